/*
 * Warp-specialised search kernels for the default decimation ladder
 * (m = 16, k = 1..6) at nharms = 60, 32 and 16: one template, one
 * configuration per harmonic count (the profile columns, the width banks of
 * each decimation and how the epilogue splits them; see Cfg60/Cfg32/Cfg16).
 *
 * One persistent CTA per SM; NIW (8 or 16) interpolation warps, then 8:
 *   warps 0..NIW-1  interpolation of harmonic blocks 0..HEAD-1 of tile i into
 *               the fp16 hi/lo A operand in tensor-memory buffer i%2 (same
 *               FP32 arithmetic as the generic kernel, bit-identical
 *               harmonic amplitudes);
 *   the last 8  the remaining harmonic blocks of tile i+1, tensor-core issue
 *               (one elected thread), then the boxcar epilogue of tile i from
 *               tensor-memory accumulator i%2.  The split evens out the two
 *               roles' instruction counts per tile.
 * Hand-off through mbarriers: a_full (one arrival per warp), a_empty and d_full
 * (tcgen05.commit).  The epilogue keeps every prefix sum in registers: with
 * the bin count and widths known at compile time, the cyclic prefix, the
 * sliding window differences P[i] - P[i-w] and the k-fold sums all unroll
 * into straight-line FP32 code in the reference's expression order.
 * Decimations k that do not divide nharms have profiles of their own (their
 * harmonic sub-stack through its own DFT columns, src/search.c:402-407),
 * scanned the same way without a fold.
 */
#pragma once

namespace wsk {

constexpr int M = 16;               /* interpolation taps */
/* interpolation warps per CTA (8 or 16; WSK_NIW* override them for tuning
 * builds); the epilogue always has 8 */
#ifndef WSK_NIW60
#define WSK_NIW60 8
#endif
#ifndef WSK_NIW32
#define WSK_NIW32 8
#endif
#ifndef WSK_NIW16
#define WSK_NIW16 8
#endif
constexpr int MAX_NH = 60;
/* tensor memory (512 columns): accumulators D0, D1 at columns 0 and 128
 * (N <= 128); operands A0, A1 (hi: K/2 columns, then lo: K/2 columns) from
 * column 256 */
constexpr int TMEM_COLS = 512;
constexpr int TM_D = 0, TM_A = 256, D_STRIDE = 128;
/* float4 stride between the tap quads of one harmonic in the weight table
 * (the largest phase-cycle length the kernels accept, so the four loads of
 * a row use immediate offsets) */
constexpr int WT_STRIDE = 128;

/* a bank of boxcar widths (src/boxcar.c:78-133), ascending */
template <int... W>
struct Widths {
    static constexpr int n = sizeof...(W);
    static __host__ __device__ constexpr int w(int a)
    {
        constexpr int v[] = {W...};
        return v[a];
    }
    static __host__ __device__ constexpr int max_w()
    {
        constexpr int v[] = {W...};
        int m = 0;
        for (int i = 0; i < n; i++) m = v[i] > m ? v[i] : m;
        return m;
    }
    static constexpr int wmax = max_w();
};

/* per-harmonic header in shared memory */
struct Harm {
    int rfloor0;
    int P;
    int woff;        /* row of phase 0 in AC */
    int wt_off;      /* float4 index of (tap quad 0, phase 0) in Wt */
    uint32_t pmagic; /* floor(2^32 / P) + 1, or 0 for P == 1 */
    int carry_res;   /* residues >= this carry into the next bin */
};

struct Args {
    const float2 *amps;
    int namps;
    const float4 *Wt;
    const float2 *A;
    const Harm *harm;
    const CsChunk *chunks;
    const int *tiles;
    int ntiles;
    const uint4 *bimg;
    int q, pnum;
    uint32_t qmagic;
    float gbound;
    const unsigned *amax;
    double thresh;
    CsRec *recs;
    unsigned *count;
    unsigned cap;
    int *err;
    /* precomputed interpolation (search_pre): X[(h - 1) * xstride + t] */
    const float2 *X;
    long long xstride;
};

template <class WS>
struct Scan {
    float hist[WS::wmax + 2];   /* hist[j] = P[i - j] */
    float mx[WS::n];
    float P, tot;
};

static __device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

template <class WS>
static __device__ __forceinline__ void scan_init(Scan<WS> &s)
{
    s.P = 0.0f;
    s.tot = 0.0f;
#pragma unroll
    for (int j = 0; j <= WS::wmax + 1; j++) s.hist[j] = 0.0f;
#pragma unroll
    for (int a = 0; a < WS::n; a++) s.mx[a] = -INFINITY;
}

/* Append profile element x as the i-th step (i = 1 .. NK + wmax) of the
 * cyclic prefix sum: P[i] = P[i-1] + x, then every window of width w ending
 * at i (start position p = i - w + 1 in 1..NK) contributes P[i] - P[i-w]
 * (src/boxcar.c:207-226).  i is a compile-time constant after unrolling. */
template <int NK, class WS>
static __device__ __forceinline__ void scan_push(Scan<WS> &s, float x, int i)
{
    s.P = __fadd_rn(s.P, x);
#pragma unroll
    for (int j = WS::wmax + 1; j > 0; j--) s.hist[j] = s.hist[j - 1];
    s.hist[0] = s.P;
    if (i == NK) s.tot = s.P;
#pragma unroll
    for (int a = 0; a < WS::n; a++) {
        const int w = WS::w(a);
        const int p = i - w + 1;
        if (p >= 1 && p <= NK) s.mx[a] = fmaxf(s.mx[a], __fsub_rn(s.hist[0], s.hist[w]));
    }
}

/* Steps i and i+1 together: both window differences of each width feed one
 * three-input max (max is exact, so the grouping does not change results). */
template <int NK, class WS>
static __device__ __forceinline__ void scan_push2(Scan<WS> &s, float x0, float x1, int i)
{
    s.P = __fadd_rn(s.P, x0);
    const float p1 = s.P;
    s.P = __fadd_rn(s.P, x1);
#pragma unroll
    for (int j = WS::wmax + 1; j > 1; j--) s.hist[j] = s.hist[j - 2];
    s.hist[1] = p1;
    s.hist[0] = s.P;
    if (i == NK) s.tot = p1;
    if (i + 1 == NK) s.tot = s.P;
#pragma unroll
    for (int a = 0; a < WS::n; a++) {
        const int w = WS::w(a);
        const int q0 = i - w + 1, q1 = q0 + 1;      /* window starts of steps i, i+1 */
        const bool v0 = q0 >= 1 && q0 <= NK, v1 = q1 >= 1 && q1 <= NK;
        const float d0 = __fsub_rn(s.hist[1], s.hist[w + 1]);
        const float d1 = __fsub_rn(s.hist[0], s.hist[w]);
        if (v0 && v1) s.mx[a] = fmax3(s.mx[a], d0, d1);
        else if (v0) s.mx[a] = fmaxf(s.mx[a], d0);
        else if (v1) s.mx[a] = fmaxf(s.mx[a], d1);
    }
}

/* max_w (M_w - duty_w * total) * invsw_w with duty_w = (float)w / (float)NK
 * (src/boxcar.c:220-228; a compile-time constant here). */
template <int NK, class WS>
static __device__ __forceinline__ float scan_finish(const Scan<WS> &s, const float *invsw)
{
    float best = -INFINITY;
#pragma unroll
    for (int a = 0; a < WS::n; a++) {
        const float duty = (float)WS::w(a) / (float)NK;
        best = fmaxf(best, __fmul_rn(__fsub_rn(s.mx[a], __fmul_rn(duty, s.tot)), invsw[a]));
    }
    return best;
}

/* The cyclic wrap: the first wmax profile elements again as steps
 * NK+1 .. NK+wmax, in pairs and a single last step when wmax is odd. */
template <int NK, class WS>
static __device__ __forceinline__ void scan_wrap(Scan<WS> &s, const float *first)
{
#pragma unroll
    for (int u = 0; u + 1 < WS::wmax; u += 2) scan_push2<NK, WS>(s, first[u], first[u + 1], NK + 1 + u);
    if (WS::wmax % 2) scan_push<NK, WS>(s, first[WS::wmax - 1], NK + WS::wmax);
}

/* Full-resolution profile: columns 0..NB-1 of the accumulator row, streamed
 * 32 columns at a time. */
template <int NB, class WS>
static __device__ __forceinline__ float base_metric(uint32_t trow, const float *invsw)
{
    static_assert(NB % 2 == 0 && NB >= WS::wmax, "profile shape");
    Scan<WS> s;
    scan_init(s);
    float first[WS::wmax];
#pragma unroll
    for (int c = 0; c < (NB + 31) / 32; c++) {
        float v[32];
        tmem_ld32(trow + 32 * c, v);
#pragma unroll
        for (int u = 0; u < 32; u += 2) {
            const int i = 32 * c + u + 1;
            if (i + 1 <= NB) {
                if (i - 1 < WS::wmax) first[i - 1] = v[u];
                if (i < WS::wmax) first[i] = v[u + 1];
                scan_push2<NB, WS>(s, v[u], v[u + 1], i);
            }
        }
    }
    scan_wrap<NB>(s, first);
    return scan_finish<NB>(s, invsw);
}

/* k-fold average of the full NB-bin profile (src/search.c:298-331): r[j] is
 * the left-to-right FP32 sum of x[j + q*NK], times (1/k), then the boxcar. */
template <int NB, int K, class WS>
static __device__ __forceinline__ float fold_metric(uint32_t trow, const float *invsw)
{
    constexpr int NK = NB / K;
    static_assert(NK * K == NB && NK % 2 == 0 && NK >= WS::wmax, "fold shape");
    float r[NK];
#pragma unroll
    for (int c = 0; c < (NB + 15) / 16; c++) {
        float v[16];
        tmem_ld16(trow + 16 * c, v);
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int i = 16 * c + u;
            if (i < NB) {
                if (i < NK) r[i % NK] = v[u];
                else r[i % NK] = __fadd_rn(r[i % NK], v[u]);
            }
        }
    }
    const float invk = 1.0f / (float)K;
    Scan<WS> s;
    scan_init(s);
#pragma unroll
    for (int j = 0; j < NK; j++) r[j] = __fmul_rn(r[j], invk);
#pragma unroll
    for (int j = 0; j < NK; j += 2) scan_push2<NK, WS>(s, r[j], r[j + 1], j + 1);
    scan_wrap<NK>(s, r);
    return scan_finish<NK>(s, invsw);
}

/* A decimation that does not fold: its own NK-bin profile in accumulator
 * columns COL0 .. COL0+NK-1 (the loads may read past it, inside the
 * accumulator's 128 columns). */
template <int COL0, int NK, class WS>
static __device__ __forceinline__ float own_metric(uint32_t trow, const float *invsw)
{
    static_assert(NK % 2 == 0 && NK >= WS::wmax && COL0 + 16 * ((NK + 15) / 16) <= D_STRIDE,
                  "profile shape");
    float r[16 * ((NK + 15) / 16)];
#pragma unroll
    for (int c = 0; c < (NK + 15) / 16; c++) tmem_ld16(trow + COL0 + 16 * c, r + 16 * c);
    Scan<WS> s;
    scan_init(s);
#pragma unroll
    for (int j = 0; j < NK; j += 2) scan_push2<NK, WS>(s, r[j], r[j + 1], j + 1);
    scan_wrap<NK>(s, r);
    return scan_finish<NK>(s, invsw);
}

static __device__ __forceinline__ void emit(const Args &a, bool hit, int ci, int slot, int j,
                                            float metric, int lane)
{
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (!mask) return;
    unsigned basei = 0;
    if (lane == 0) basei = atomicAdd(a.count, (unsigned)__popc(mask));
    basei = __shfl_sync(0xffffffffu, basei, 0);
    if (hit) {
        const unsigned pos = basei + (unsigned)__popc(mask & ((1u << lane) - 1u));
        if (pos < a.cap) {
            CsRec rec;
            rec.chunk = ci;
            rec.slot = slot;
            rec.j = j;
            rec.metric = metric;
            a.recs[pos] = rec;
        }
    }
}

/* 4 consecutive 32-bit tensor-memory columns of this warp's 32 lanes */
static __device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b,
                                                uint32_t c, uint32_t d)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};"
                 :: "r"(taddr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

/* D[tmem] (+)= A[tmem] * B[smem]^T, 128 x N x 16, fp16 in, fp32 accumulate */
static __device__ __forceinline__ void mma_f16_ts(uint32_t d_tmem, uint32_t a_tmem,
                                                  uint64_t bdesc, uint32_t idesc,
                                                  uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

static __device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}

/* barrier over the 256 epilogue threads with an AND vote */
static __device__ __forceinline__ bool epi_bar_and(bool v)
{
    uint32_t out;
    asm volatile("{\n\t.reg .pred p, q;\n\t"
                 "setp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.and.pred q, 1, 256, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(out) : "r"((uint32_t)v) : "memory");
    return out != 0;
}

static __device__ __forceinline__ uint32_t mod_magic(uint32_t t, uint32_t P, uint32_t magic)
{
    if (P == 1) return 0;
    uint32_t e = __umulhi(t, magic);
    uint32_t pr = e * P;
    if (pr > t) pr -= P;
    return t - pr;
}



struct TrialState {
    uint32_t t, Q, R;               /* trial index, t*pnum = Q*q + R */
    bool valid;
    unsigned long long filled;
};

static __device__ __forceinline__ TrialState trial_state(const Args &a, int tile, int r)
{
    TrialState ts;
    const int ci = a.tiles[3 * tile], j0 = a.tiles[3 * tile + 1];
    const int cnt = a.tiles[3 * tile + 2];
    const CsChunk &ch = a.chunks[ci];
    ts.filled = ch.filled;
    ts.valid = r < cnt;
    ts.t = (uint32_t)(ch.i0 + j0 + r);
    if (a.pnum == 1) {
        divmod_q(ts.t, (uint32_t)a.q, a.qmagic, ts.Q, ts.R);
    } else {
        const unsigned long long tp = (unsigned long long)ts.t * (unsigned)a.pnum;
        ts.Q = (uint32_t)(tp / (unsigned)a.q);
        ts.R = (uint32_t)(tp - (unsigned long long)ts.Q * (unsigned)a.q);
    }
    return ts;
}

/* residue and quotient of t*h*pnum over q (h <= 60, so h*R < 2^32) */
static __device__ __forceinline__ void state_at(const Args &a, const TrialState &ts, uint32_t h,
                                                uint32_t &res, uint32_t &qint)
{
    uint32_t qd;
    divmod_q(h * ts.R, (uint32_t)a.q, a.qmagic, qd, res);
    qint = h * ts.Q + qd;
}

/* Interpolate harmonics 4hb+1..4hb+4 of one trial (src/cuda.cu:120-135
 * arithmetic) and store them, split into fp16 hi/lo, as K block hb of the
 * A operand in tensor memory.  (res, qint) enter at h = 4hb+1 and leave at
 * h = 4hb+5. */
/* Store 4 harmonics of one trial, scaled and split into fp16 hi/lo, as K
 * block hb of the A operand in tensor memory. */
template <int AHALF>
static __device__ __forceinline__ void store_block(const float *xr4, const float *xi4, float scale,
                                                   int hb, uint32_t abuf)
{
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const float2 sc = make_float2(xr4[u] * scale, xi4[u] * scale);
        const __half2 hi = __float22half2_rn(sc);
        const float2 back = __half22float2(hi);
        const __half2 lo = __float22half2_rn(
            make_float2(__fsub_rn(sc.x, back.x), __fsub_rn(sc.y, back.y)));
        hw[u] = *reinterpret_cast<const uint32_t *>(&hi);
        lw[u] = *reinterpret_cast<const uint32_t *>(&lo);
    }
    /* K block hb = columns 4hb..4hb+3 (two halves per column); lo K/2 columns on */
    tmem_st4(abuf + 4 * hb, hw[0], hw[1], hw[2], hw[3]);
    tmem_st4(abuf + AHALF + 4 * hb, lw[0], lw[1], lw[2], lw[3]);
}

template <int AHALF>
static __device__ __forceinline__ void interp_block(const Args &a, const Harm *hs,
                                                    const TrialState &ts, int hb,
                                                    uint32_t &res, uint32_t &qint,
                                                    float scale, uint32_t abuf)
{
    const uint32_t t = ts.t, R = ts.R, Q = ts.Q;
    const bool full = ts.valid && (((ts.filled >> (4 * hb)) & 0xFULL) == 0xFULL);
    float xr4[4], xi4[4];
    if (full) {
        /* every harmonic of the block is active: no branches, so the loads of
         * all four harmonics can be in flight together */
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const Harm hm = hs[4 * hb + u];
            const uint32_t ph = mod_magic(t, (uint32_t)hm.P, hm.pmagic);
            const int b0 = hm.rfloor0 + (int)qint + ((int)res >= hm.carry_res ? 1 : 0) + 1 - M / 2;
            /* in range by construction for active harmonics; clamp for safety */
            const int bs = min(max(b0, 0), a.namps - M);
            const float2 *ap = a.amps + bs;
            const float4 *wq = a.Wt + hm.wt_off + ph;
            /* packed FP32: each lane of __ffma2_rn is a correctly rounded fma,
             * so (Re, Im) advance exactly as two scalar chains */
            float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int i4 = 0; i4 < M / 4; i4++) {
                const float4 w = __ldg(wq + i4 * WT_STRIDE);
                const float2 v0 = __ldg(ap + 4 * i4), v1 = __ldg(ap + 4 * i4 + 1);
                const float2 v2 = __ldg(ap + 4 * i4 + 2), v3 = __ldg(ap + 4 * i4 + 3);
                acc = __ffma2_rn(make_float2(w.x, w.x), v0, acc);
                acc = __ffma2_rn(make_float2(w.y, w.y), v1, acc);
                acc = __ffma2_rn(make_float2(w.z, w.z), v2, acc);
                acc = __ffma2_rn(make_float2(w.w, w.w), v3, acc);
            }
            const float2 g = __ldg(a.A + hm.woff + ph);
            const bool inb = (b0 == bs);
            xr4[u] = inb ? __fsub_rn(__fmul_rn(g.x, acc.x), __fmul_rn(g.y, acc.y)) : 0.0f;
            xi4[u] = inb ? __fadd_rn(__fmul_rn(g.x, acc.y), __fmul_rn(g.y, acc.x)) : 0.0f;
            res += R; qint += Q;
            if (res >= (uint32_t)a.q) { res -= (uint32_t)a.q; qint += 1; }
        }
    } else {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int h = 4 * hb + u + 1;
            float xr = 0.0f, xi = 0.0f;
            if (ts.valid && ((ts.filled >> (h - 1)) & 1ULL)) {
                const Harm hm = hs[h - 1];
                const uint32_t ph = mod_magic(t, (uint32_t)hm.P, hm.pmagic);
                const int b0 = hm.rfloor0 + (int)qint + ((int)res >= hm.carry_res ? 1 : 0) + 1 - M / 2;
                float ar = 0.0f, ai = 0.0f;
                if ((unsigned)b0 <= (unsigned)(a.namps - M)) {
                    const float2 *ap = a.amps + b0;
                    const float4 *wq = a.Wt + hm.wt_off + ph;
#pragma unroll
                    for (int i4 = 0; i4 < M / 4; i4++) {
                        const float4 w = __ldg(wq + i4 * WT_STRIDE);
                        const float2 v0 = __ldg(ap + 4 * i4), v1 = __ldg(ap + 4 * i4 + 1);
                        const float2 v2 = __ldg(ap + 4 * i4 + 2), v3 = __ldg(ap + 4 * i4 + 3);
                        ar = __fmaf_rn(w.x, v0.x, ar); ai = __fmaf_rn(w.x, v0.y, ai);
                        ar = __fmaf_rn(w.y, v1.x, ar); ai = __fmaf_rn(w.y, v1.y, ai);
                        ar = __fmaf_rn(w.z, v2.x, ar); ai = __fmaf_rn(w.z, v2.y, ai);
                        ar = __fmaf_rn(w.w, v3.x, ar); ai = __fmaf_rn(w.w, v3.y, ai);
                    }
                }
                const float2 g = __ldg(a.A + hm.woff + ph);
                xr = __fsub_rn(__fmul_rn(g.x, ar), __fmul_rn(g.y, ai));
                xi = __fadd_rn(__fmul_rn(g.x, ai), __fmul_rn(g.y, ar));
            }
            xr4[u] = xr;
            xi4[u] = xi;
            res += R; qint += Q;
            if (res >= (uint32_t)a.q) { res -= (uint32_t)a.q; qint += 1; }
        }
    }
    store_block<AHALF>(xr4, xi4, scale, hb, abuf);
}

/* Threshold one metric of slot S of this row (warp-aggregated compaction). */
template <int S>
static __device__ __forceinline__ void post(const Args &a, const CsChunk &ch, float m, bool valid,
                                            int ci, int j, int lane)
{
    emit(a, valid && j < ch.nvalid[S] && (double)m > a.thresh, ci, S, j, m, lane);
}

using W5 = Widths<1, 2, 3, 4, 6>;
using W4 = Widths<2, 3, 4, 6>;
using W3 = Widths<2, 3, 4>;
using W2 = Widths<2, 3>;

/* Per harmonic count: MMA shape (N = profile columns, K = 2*nharms padded),
 * the split of harmonic blocks between the roles (blocks 0..HEAD-1 on the
 * interpolation warps, HEAD..HEAD+G0-1 on epilogue group 0, the rest on
 * group 1) and the epilogue.  Slots are in the host tables' order: k = 1,
 * then k = 2..6; a k that does not divide nharms has its own profile columns
 * after the 2*nharms of the base profile (cs_tables.c), at the offsets and
 * with the width banks (src/boxcar.c:100-133) written out below.  Each
 * group's epilogue work is balanced against its share of the blocks. */
struct Cfg60 {
    static constexpr int NH = 60, NPAD = 128, KPAD = 128, HEAD = 12, G0 = 2, NIW = WSK_NIW60;
    static __device__ __forceinline__ void epilogue(int grp, uint32_t trow, const CsChunk &ch,
                                                    const Args &a, bool valid, int ci, int j,
                                                    int lane, float inv)
    {
        if (grp == 0) {
            post<0>(a, ch, base_metric<120, W5>(trow, ch.invsw[0]) * inv, valid, ci, j, lane);
            post<5>(a, ch, fold_metric<120, 6, W4>(trow, ch.invsw[5]) * inv, valid, ci, j, lane);
        } else {
            post<1>(a, ch, fold_metric<120, 2, W4>(trow, ch.invsw[1]) * inv, valid, ci, j, lane);
            post<2>(a, ch, fold_metric<120, 3, W4>(trow, ch.invsw[2]) * inv, valid, ci, j, lane);
            post<3>(a, ch, fold_metric<120, 4, W4>(trow, ch.invsw[3]) * inv, valid, ci, j, lane);
            post<4>(a, ch, fold_metric<120, 5, W4>(trow, ch.invsw[4]) * inv, valid, ci, j, lane);
        }
    }
    /* the same slots over four groups (search_pre): the base profile alone,
     * then the folds paired by cost */
    static __device__ __forceinline__ void epilogue4(int grp, uint32_t trow, const CsChunk &ch,
                                                     const Args &a, bool valid, int ci, int j,
                                                     int lane, float inv)
    {
        if (grp == 0) {
            post<0>(a, ch, base_metric<120, W5>(trow, ch.invsw[0]) * inv, valid, ci, j, lane);
        } else if (grp == 1) {
            post<1>(a, ch, fold_metric<120, 2, W4>(trow, ch.invsw[1]) * inv, valid, ci, j, lane);
            post<5>(a, ch, fold_metric<120, 6, W4>(trow, ch.invsw[5]) * inv, valid, ci, j, lane);
        } else if (grp == 2) {
            post<2>(a, ch, fold_metric<120, 3, W4>(trow, ch.invsw[2]) * inv, valid, ci, j, lane);
            post<4>(a, ch, fold_metric<120, 5, W4>(trow, ch.invsw[4]) * inv, valid, ci, j, lane);
        } else {
            post<3>(a, ch, fold_metric<120, 4, W4>(trow, ch.invsw[3]) * inv, valid, ci, j, lane);
        }
    }
};

struct Cfg32 {
    static constexpr int NH = 32, NPAD = 112, KPAD = 64, HEAD = 6, G0 = 1, NIW = WSK_NIW32;
    static __device__ __forceinline__ void epilogue(int grp, uint32_t trow, const CsChunk &ch,
                                                    const Args &a, bool valid, int ci, int j,
                                                    int lane, float inv)
    {
        if (grp == 0) {
            post<0>(a, ch, base_metric<64, W5>(trow, ch.invsw[0]) * inv, valid, ci, j, lane);
            post<4>(a, ch, own_metric<84, 12, W2>(trow, ch.invsw[4]) * inv, valid, ci, j, lane);
            post<5>(a, ch, own_metric<96, 10, W2>(trow, ch.invsw[5]) * inv, valid, ci, j, lane);
        } else {
            post<1>(a, ch, fold_metric<64, 2, W4>(trow, ch.invsw[1]) * inv, valid, ci, j, lane);
            post<2>(a, ch, own_metric<64, 20, W4>(trow, ch.invsw[2]) * inv, valid, ci, j, lane);
            post<3>(a, ch, fold_metric<64, 4, W3>(trow, ch.invsw[3]) * inv, valid, ci, j, lane);
        }
    }
};

struct Cfg16 {
    static constexpr int NH = 16, NPAD = 64, KPAD = 32, HEAD = 3, G0 = 1, NIW = WSK_NIW16;
    static __device__ __forceinline__ void epilogue(int grp, uint32_t trow, const CsChunk &ch,
                                                    const Args &a, bool valid, int ci, int j,
                                                    int lane, float inv)
    {
        if (grp == 0) {
            post<0>(a, ch, base_metric<32, W5>(trow, ch.invsw[0]) * inv, valid, ci, j, lane);
            post<5>(a, ch, own_metric<48, 4, Widths<1>>(trow, ch.invsw[5]) * inv, valid, ci, j,
                    lane);
        } else {
            post<1>(a, ch, fold_metric<32, 2, W3>(trow, ch.invsw[1]) * inv, valid, ci, j, lane);
            post<2>(a, ch, own_metric<32, 10, W2>(trow, ch.invsw[2]) * inv, valid, ci, j, lane);
            post<3>(a, ch, fold_metric<32, 4, Widths<2>>(trow, ch.invsw[3]) * inv, valid, ci, j,
                    lane);
            post<4>(a, ch, own_metric<42, 6, Widths<1>>(trow, ch.invsw[4]) * inv, valid, ci, j,
                    lane);
        }
    }
};

/* The same layouts for the host's check that a session's tables are the
 * ones a configuration was compiled for. */
struct SlotDesc {
    int k, nk, fold, col0, nw, w[6];
};
struct CfgDesc {
    int nh, npad, kpad;
    SlotDesc slot[6];
};
static const CfgDesc kCfgDescs[3] = {
    {60, 128, 128, {{1, 120, 0, 0, 5, {1, 2, 3, 4, 6}}, {2, 60, 1, -1, 4, {2, 3, 4, 6}},
                    {3, 40, 1, -1, 4, {2, 3, 4, 6}}, {4, 30, 1, -1, 4, {2, 3, 4, 6}},
                    {5, 24, 1, -1, 4, {2, 3, 4, 6}}, {6, 20, 1, -1, 4, {2, 3, 4, 6}}}},
    {32, 112, 64, {{1, 64, 0, 0, 5, {1, 2, 3, 4, 6}}, {2, 32, 1, -1, 4, {2, 3, 4, 6}},
                   {3, 20, 0, 64, 4, {2, 3, 4, 6}}, {4, 16, 1, -1, 3, {2, 3, 4}},
                   {5, 12, 0, 84, 2, {2, 3}}, {6, 10, 0, 96, 2, {2, 3}}}},
    {16, 64, 32, {{1, 32, 0, 0, 5, {1, 2, 3, 4, 6}}, {2, 16, 1, -1, 3, {2, 3, 4}},
                  {3, 10, 0, 32, 2, {2, 3}}, {4, 8, 1, -1, 1, {2}},
                  {5, 6, 0, 42, 1, {1}}, {6, 4, 0, 48, 1, {1}}}},
};

template <class C>
__host__ __device__ constexpr int nthreads()
{
    return (C::NIW + 8) * 32;
}

template <class C>
__host__ __device__ constexpr int smem_bytes()
{
    return 2 * C::NPAD * C::KPAD * 2 + 64 + 16 + C::NH * (int)sizeof(Harm);
}

/* the multi-spectrum kernel adds one header slot per warp */
template <class C>
__host__ __device__ constexpr int smem_bytes_multi()
{
    return smem_bytes<C>() + (C::NIW + 8) * C::NH * (int)sizeof(Harm);
}

/* Several spectra of the same configuration in one persistent launch: a
 * table of per-spectrum arguments (c_multi_files) and the prefix sums of
 * their tile counts (c_multi_off).  Each tile takes its spectrum's tables,
 * operand scale and record buffer.
 *
 * Schedule: rounds of grid x `block` consecutive tiles of the concatenated
 * list; in each round CTA b takes the b-th block of `block` tiles, and the
 * last, partial round is split evenly (to one tile) over the CTAs.  At any
 * time every CTA works inside the same few spectra, so the L2 holds their
 * windows and weight rows as it does for one spectrum (CTA-contiguous runs
 * over a long list put every CTA in a different spectrum, a working set of
 * many spectra); within a block neighbouring tiles still share L1 lines. */
struct Multi {
    int nfiles;
    int ntiles;
    int block;
};

/* Both tables live in constant memory.  Every index into them is uniform
 * over the CTA (derived from the tile loop and the tables alone), so the
 * per-spectrum fields are broadcast reads held in uniform registers, as
 * cheap as kernel parameters, and stay off the L1 load path the
 * interpolation is bound on.  Launches on one device are serialised by the
 * host. */
constexpr int MULTI_MAX = 400;
__constant__ Args c_multi_files[MULTI_MAX];
__constant__ int c_multi_off[MULTI_MAX + 1];

/* A role's walk over its CTA's tiles: g the global tile, end the end of the
 * current run (single spectrum: the CTA's contiguous run; several: the
 * current block), f the spectrum of g.  Tiles come in increasing order, so
 * f only moves forward. */
struct Walk {
    int g, end, f, base;
};

/* The CTA's block of the round starting at tile w.base (false: none). */
static __device__ __forceinline__ bool walk_block(Walk &w, const Multi &mu)
{
    const int G = (int)gridDim.x, b = (int)blockIdx.x;
    if (w.base >= mu.ntiles) return false;
    const int rem = mu.ntiles - w.base;
    if (rem >= G * mu.block) {
        w.g = w.base + b * mu.block;
        w.end = w.g + mu.block;
    } else {
        w.g = w.base + (int)(((long long)b * rem) / G);
        w.end = w.base + (int)(((long long)(b + 1) * rem) / G);
    }
    return w.g < w.end;
}

template <bool MULTI>
static __device__ __forceinline__ bool walk_begin(Walk &w, const Multi &mu, int tile_begin,
                                                  int tile_end)
{
    w.f = 0;
    if (!MULTI) {
        w.g = tile_begin;
        w.end = tile_end;
        return w.g < w.end;
    }
    w.base = 0;
    return walk_block(w, mu);
}

template <bool MULTI>
static __device__ __forceinline__ bool walk_next(Walk &w, const Multi &mu)
{
    if (++w.g < w.end) return true;
    if (!MULTI) return false;
    w.base += (int)gridDim.x * mu.block;
    return walk_block(w, mu);
}

/* The local tile index of the walk's tile; moves w.f to its spectrum. */
template <bool MULTI>
static __device__ __forceinline__ int walk_tile(Walk &w)
{
    if (!MULTI) return w.g;
    while (w.g >= c_multi_off[w.f + 1]) w.f++;
    return w.g - c_multi_off[w.f];
}

/* A warp's private copy of spectrum f's harmonic headers (shared memory,
 * refreshed when the warp's walk enters another spectrum; no other warp
 * reads it, so a __syncwarp on both sides orders it). */
template <int NH>
static __device__ __forceinline__ void load_headers(Harm *slot, int f, int lane)
{
    __syncwarp();
    const int *src = reinterpret_cast<const int *>(c_multi_files[f].harm);
    int *dst = reinterpret_cast<int *>(slot);
    constexpr int NW = NH * (int)sizeof(Harm) / 4;
    for (int i = lane; i < NW; i += 32) dst[i] = __ldg(src + i);
    __syncwarp();
}

/* The arguments of a tile: the launch's own, or (MULTI) its spectrum's entry
 * of the constant table.  For nharms 60 the entry is copied out once per
 * tile, so that the fields the harmonic loop reads sit in registers instead
 * of being re-read from the table inside it (measured: 1.63 -> 1.68 G
 * trials/s); the smaller configurations run faster reading the table
 * (their extra registers cost more than the reads).  Bit k of
 * WSK_MULTI_COPY selects the copy for configuration k (16, 32, 60). */
#ifndef WSK_MULTI_COPY
#define WSK_MULTI_COPY 4
#endif
#define WS_TILE_ARGS(a, f)                                                       \
    constexpr bool a##_cp = MULTI && ((WSK_MULTI_COPY >> (NH == 16 ? 0 : NH == 32 ? 1 : 2)) & 1); \
    Args a##_copy;                                                               \
    if constexpr (a##_cp) a##_copy = c_multi_files[(f)];                         \
    const Args &a = a##_cp ? a##_copy : MULTI ? c_multi_files[(f)] : a0

/* A failed wait: every spectrum of the launch reports the error. */
template <bool MULTI>
static __device__ __forceinline__ void set_err(const Args &a0, const Multi &mu)
{
    if constexpr (!MULTI) {
        atomicExch(a0.err, 1);
    } else {
        for (int f = 0; f < mu.nfiles; f++) atomicExch(c_multi_files[f].err, 1);
    }
}

template <class C, bool MULTI>
static __device__ __forceinline__ void ws_body(const Args &a0, const Multi &mu)
{
    constexpr int NH = C::NH, NPAD = C::NPAD, KPAD = C::KPAD, AHALF = KPAD / 2;
    constexpr int NIW = C::NIW, NPAR = NIW / 4, NTHREADS = nthreads<C>();
    static_assert(NIW == 8 || NIW == 16, "interpolation warps");
    constexpr int HEAD = C::HEAD, G0 = C::G0;
    constexpr int BIMG = NPAD * KPAD * 2;            /* one fp16 B image */
    /* shared memory: B hi/lo | barriers | tmem slot | harmonic headers; the
     * rest of the SM's 256 KB stays L1 for the weight and spectrum reads */
    constexpr int SM_B = 0, SM_BAR = 2 * BIMG, SM_TM = SM_BAR + 64, SM_HARM = SM_TM + 16;
    static_assert(SM_HARM + NH * (int)sizeof(Harm) == smem_bytes<C>(), "layout");
    static_assert(NH % 4 == 0 && 2 * NH <= KPAD && KPAD % 16 == 0 && NPAD <= D_STRIDE &&
                  NPAD % 16 == 0 && HEAD + G0 <= NH / 4, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar_afull = smem_u32(smem + SM_BAR);        /* 2 x 8 B */
    const uint32_t bar_aempty = bar_afull + 16;
    const uint32_t bar_dfull = bar_afull + 32;
    uint32_t *tm_slot = reinterpret_cast<uint32_t *>(smem + SM_TM);
    Harm *hs = reinterpret_cast<Harm *>(smem + SM_HARM);
    Harm *hslot = hs + NH * (1 + warp);              /* MULTI: this warp's headers */
    /* one spectrum: each CTA owns a contiguous run of tiles (neighbouring
     * tiles read the same spectral windows and weight rows, which then stay
     * in L1); several: the block-cyclic walk of struct Multi */
    const int per_cta = (a0.ntiles + gridDim.x - 1) / gridDim.x;
    const int tile_begin = MULTI ? 0 : min(a0.ntiles, (int)blockIdx.x * per_cta);
    const int tile_end = MULTI ? 0 : min(a0.ntiles, tile_begin + per_cta);

    if (warp == 0) tmem_alloc(smem_u32(tm_slot), TMEM_COLS);
    if (!MULTI)
        for (int h = tid; h < NH; h += NTHREADS) hs[h] = a0.harm[h];
    if (tid == 0) {
        mbar_init(bar_afull, NIW + 8);      /* every interpolation and epilogue warp */
        mbar_init(bar_afull + 8, NIW + 8);
        mbar_init(bar_aempty, 1);
        mbar_init(bar_aempty + 8, 1);
        mbar_init(bar_dfull, 1);
        mbar_init(bar_dfull + 8, 1);
    }
    {
        uint4 *dst = reinterpret_cast<uint4 *>(smem + SM_B);
        for (int i = tid; i < (2 * BIMG) / 16; i += NTHREADS) dst[i] = a0.bimg[i];
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tm_slot;
    /* the fp16 operand scale of a spectrum (one per launch unless MULTI) */
    const float scale0 = MULTI ? 1.0f : operand_scale(a0.amax, a0.gbound);
    if (warp < NIW) {
        /* --------------- interpolation of blocks 0..HEAD-1 --------------- */
        const int r = tid & (CS_TILE_M - 1);
        const int par = tid >> 7;
        const uint32_t tlane = (uint32_t)((warp & 3) * 32) << 16;
        if (par == 1) {
            /* the K padding columns (harmonics past nharms) of both A buffers stay zero */
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const uint32_t ab = tmem + tlane + (uint32_t)(TM_A + KPAD * b);
#pragma unroll
                for (int c = NH; c < AHALF; c += 4) {
                    tmem_st4(ab + c, 0, 0, 0, 0);
                    tmem_st4(ab + AHALF + c, 0, 0, 0, 0);
                }
            }
        }
        Walk w;
        int fcur = -1;
        float scale = scale0;
        bool more = walk_begin<MULTI>(w, mu, tile_begin, tile_end);
        for (int it = 0; more; it++, more = walk_next<MULTI>(w, mu)) {
            const int s = it & 1;
            if (it >= 2 && !mbar_wait(bar_aempty + 8 * s, ((it - 2) >> 1) & 1)) {
                if (lane == 0) set_err<MULTI>(a0, mu);
                break;
            }
            tc_fence_after();
            const int tile = walk_tile<MULTI>(w);
            WS_TILE_ARGS(a, w.f);
            if (MULTI && w.f != fcur) {
                fcur = w.f;
                load_headers<NH>(hslot, fcur, lane);
                scale = operand_scale(a.amax, a.gbound);
            }
            const Harm *hsp = MULTI ? hslot : hs;
            const TrialState ts = trial_state(a, tile, r);
            const uint32_t abuf = tmem + tlane + (uint32_t)(TM_A + KPAD * s);
            uint32_t res, qint, r4, q4;
            state_at(a, ts, 4u * par + 1u, res, qint);
            state_at(a, ts, 4u * (NPAR - 1), r4, q4);   /* the harmonics other groups take */
            for (int hb = par; hb < HEAD; hb += NPAR) {
                interp_block<AHALF>(a, hsp, ts, hb, res, qint, scale, abuf);
                res += r4; qint += q4;       /* 4hb+5 -> 4(hb+NPAR)+1 */
                if (res >= (uint32_t)a.q) { res -= (uint32_t)a.q; qint += 1; }
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_afull + 8 * s);
        }
    } else {
        /* ----- tensor cores, epilogue, and blocks HEAD.. of the next tile ---- */
        const int e = warp - NIW;
        const int quarter = e & 3, grp = e >> 2;
        const int r = quarter * 32 + lane;
        const uint32_t tlane = (uint32_t)(quarter * 32) << 16;
        const bool leader = (warp == NIW && lane == 0);
        const uint32_t idesc = (1u << 4) | ((uint32_t)(NPAD >> 3) << 17) |
                               ((uint32_t)(CS_TILE_M >> 4) << 24);
        const uint32_t lbo_b = NPAD * 16;
        const uint32_t b_hi = smem_u32(smem + SM_B), b_lo = b_hi + BIMG;
        /* tail blocks: group 0 has the lighter epilogue and takes more of them */
        const int tb0 = grp == 0 ? HEAD : HEAD + G0;
        const int tb1 = grp == 0 ? HEAD + G0 : NH / 4;
        int issued = 0, consumed = 0;
        bool ok = true;

        /* walks of the tail blocks (one tile ahead) and of the epilogue, with
         * the spectrum and operand scale each last saw */
        Walk wt, we;
        int ft_cur = -1, fe_cur = -1;
        float scale_t = scale0, inv_scale = 1.0f / scale0;
        auto tail = [&](int it) {
            const int tile = walk_tile<MULTI>(wt);
            WS_TILE_ARGS(a, wt.f);
            if (MULTI && wt.f != ft_cur) {
                ft_cur = wt.f;
                load_headers<NH>(hslot, ft_cur, lane);
                scale_t = operand_scale(a.amax, a.gbound);
            }
            const Harm *hsp = MULTI ? hslot : hs;
            const float scale = scale_t;
            const TrialState ts = trial_state(a, tile, r);
            const uint32_t abuf = tmem + tlane + (uint32_t)(TM_A + KPAD * (it & 1));
            uint32_t res, qint;
            state_at(a, ts, 4u * tb0 + 1u, res, qint);
            for (int hb = tb0; hb < tb1; hb++)
                interp_block<AHALF>(a, hsp, ts, hb, res, qint, scale, abuf);
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_afull + 8 * (it & 1));
        };
        auto issue = [&](int it) -> bool {
            const int s = it & 1;
            if (!mbar_wait(bar_afull + 8 * s, (it >> 1) & 1)) return false;
            tc_fence_after();
            const uint32_t a_hi = tmem + (uint32_t)(TM_A + KPAD * s), a_lo = a_hi + AHALF;
            const uint32_t d = tmem + (uint32_t)(TM_D + D_STRIDE * s);
            uint32_t acc = 0;
#pragma unroll
            for (int pass = 0; pass < 3; pass++) {
                const uint32_t abase = (pass == 1) ? a_lo : a_hi;
                const uint32_t bbase = (pass == 2) ? b_lo : b_hi;
#pragma unroll
                for (int k = 0; k < KPAD / 16; k++) {
                    mma_f16_ts(d, abase + (uint32_t)(8 * k),
                               umma_desc(bbase + (uint32_t)k * 2 * lbo_b, lbo_b, 128), idesc, acc);
                    acc = 1;
                }
            }
            mma_commit(bar_aempty + 8 * s);
            mma_commit(bar_dfull + 8 * s);
            return true;
        };

        /* tile 0: its tail blocks, then its MMAs */
        bool tmore = walk_begin<MULTI>(wt, mu, tile_begin, tile_end);
        bool emore = walk_begin<MULTI>(we, mu, tile_begin, tile_end);
        if (tmore) {
            tail(0);
            if (leader) {
                ok = issue(0);
                if (ok) issued = 1;
                else set_err<MULTI>(a0, mu);
            }
            __syncwarp();
        }
        for (int it = 0; emore; it++, emore = walk_next<MULTI>(we, mu)) {
            const int s = it & 1;
            tmore = tmore && walk_next<MULTI>(wt, mu);
            if (tmore) {
                /* A buffer (it+1)&1 was last read by the MMA of tile it-1, whose
                 * accumulator this group already consumed: it is free */
                tail(it + 1);
                if (leader && ok) {
                    ok = issue(it + 1);
                    if (ok) issued++;
                    else set_err<MULTI>(a0, mu);
                }
                __syncwarp();
            }
            bool got = mbar_wait(bar_dfull + 8 * s, (it >> 1) & 1);
            if (!epi_bar_and(got && ok)) {
                if (lane == 0) set_err<MULTI>(a0, mu);
                ok = false;
                break;
            }
            consumed++;
            tc_fence_after();
            const int tile = walk_tile<MULTI>(we);
            /* the epilogue reads few fields: a reference into the table */
            const Args &a = MULTI ? c_multi_files[we.f] : a0;
            if (MULTI && we.f != fe_cur) {
                fe_cur = we.f;
                inv_scale = 1.0f / operand_scale(a.amax, a.gbound);
            }
            const int ci = a.tiles[3 * tile], j0 = a.tiles[3 * tile + 1];
            const int cnt = a.tiles[3 * tile + 2];
            const CsChunk &ch = a.chunks[ci];
            const bool valid = r < cnt;
            const int j = j0 + r;
            const uint32_t trow = tmem + (uint32_t)(TM_D + s * D_STRIDE) + ((uint32_t)(quarter * 32) << 16);
            C::epilogue(grp, trow, ch, a, valid, ci, j, lane, inv_scale);
            tc_fence_before();
            epi_bar_and(true);      /* accumulator s free for the MMA of tile it+2 */
        }
        /* drain: never free tensor memory under an MMA in flight */
        if (leader) {
            for (int k = consumed; k < issued; k++)
                mbar_wait(bar_dfull + 8 * (k & 1), (k >> 1) & 1);
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

template <class C>
__global__ void __launch_bounds__(nthreads<C>(), 1) search_ws(const __grid_constant__ Args a)
{
    const Multi none = {0, 0, 1};
    ws_body<C, false>(a, none);
}

/* The search with the interpolated values precomputed (X[h][t], by the
 * tensor-core interpolation tci::interp_tc): all 16 warps in lockstep.
 * Warp w owns trial rows 32 (w & 3) .. of a tile and group w >> 2.  Per
 * tile it: load X of tile it + 2 (blocks g, g + 4, ... of the warp's rows),
 * wait for the transform of tile it, run epilogue group g on it, store the
 * loaded values as tile it + 2's A operand (its A buffer is free once the
 * transform of tile it is done), barrier, then one thread issues the
 * transform of tile it + 2.  Two transforms stay in flight behind the
 * epilogue. */
template <class C>
static __device__ __forceinline__ void pre_body(const Args &a)
{
    constexpr int NH = C::NH, NPAD = C::NPAD, KPAD = C::KPAD, AHALF = KPAD / 2;
    constexpr int NBLK = NH / 4;                       /* K blocks of 4 harmonics */
    constexpr int JB = (NBLK + 3) / 4;                 /* blocks a warp */
    constexpr int BIMG = NPAD * KPAD * 2;
    constexpr int SM_B = 0, SM_BAR = 2 * BIMG, SM_TM = SM_BAR + 64;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, grp = warp >> 2;
    const int r = quarter * 32 + lane;
    const uint32_t tlane = (uint32_t)(quarter * 32) << 16;
    const uint32_t bar_d = smem_u32(smem + SM_BAR);               /* 2 x 8 B */
    uint32_t *tm_slot = reinterpret_cast<uint32_t *>(smem + SM_TM);
    const int per_cta = (a.ntiles + gridDim.x - 1) / gridDim.x;
    const int tile_begin = min(a.ntiles, (int)blockIdx.x * per_cta);
    const int ntl = min(a.ntiles, tile_begin + per_cta) - tile_begin;

    if (warp == 0) tmem_alloc(smem_u32(tm_slot), TMEM_COLS);
    if (tid == 0) {
        mbar_init(bar_d, 1);
        mbar_init(bar_d + 8, 1);
    }
    {
        uint4 *dst = reinterpret_cast<uint4 *>(smem + SM_B);
        for (int i = tid; i < (2 * BIMG) / 16; i += blockDim.x) dst[i] = a.bimg[i];
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tm_slot;
    const float scale = operand_scale(a.amax, a.gbound);
    const float inv_scale = 1.0f / scale;
    const uint32_t idesc = (1u << 4) | ((uint32_t)(NPAD >> 3) << 17) |
                           ((uint32_t)(CS_TILE_M >> 4) << 24);
    const uint32_t lbo_b = NPAD * 16;
    const uint32_t b_hi = smem_u32(smem + SM_B), b_lo = b_hi + BIMG;

    /* X of tile index i (0-based in the CTA's run) for the warp's blocks */
    auto load_x = [&](int i, float2 (&xv)[JB][4]) {
        const TrialState ts = trial_state(a, tile_begin + i, r);
#pragma unroll
        for (int jb = 0; jb < JB; jb++) {
            const int hb = grp + 4 * jb;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int h = 4 * hb + u + 1;
                xv[jb][u] = (hb < NBLK && ts.valid && ((ts.filled >> (h - 1)) & 1ULL))
                                ? __ldg(a.X + (long long)(h - 1) * a.xstride + ts.t)
                                : make_float2(0.0f, 0.0f);
            }
        }
    };
    auto store_a = [&](int s, const float2 (&xv)[JB][4]) {
        const uint32_t abuf = tmem + tlane + (uint32_t)(TM_A + KPAD * s);
#pragma unroll
        for (int jb = 0; jb < JB; jb++) {
            const int hb = grp + 4 * jb;
            if (hb >= NBLK) break;
            const float xr4[4] = {xv[jb][0].x, xv[jb][1].x, xv[jb][2].x, xv[jb][3].x};
            const float xi4[4] = {xv[jb][0].y, xv[jb][1].y, xv[jb][2].y, xv[jb][3].y};
            store_block<AHALF>(xr4, xi4, scale, hb, abuf);
        }
    };
    auto issue = [&](int s) {
        const uint32_t a_hi = tmem + (uint32_t)(TM_A + KPAD * s), a_lo = a_hi + AHALF;
        const uint32_t d = tmem + (uint32_t)(TM_D + D_STRIDE * s);
        uint32_t acc = 0;
#pragma unroll
        for (int pass = 0; pass < 3; pass++) {
            const uint32_t abase = (pass == 1) ? a_lo : a_hi;
            const uint32_t bbase = (pass == 2) ? b_lo : b_hi;
#pragma unroll
            for (int k = 0; k < KPAD / 16; k++) {
                mma_f16_ts(d, abase + (uint32_t)(8 * k),
                           umma_desc(bbase + (uint32_t)k * 2 * lbo_b, lbo_b, 128), idesc, acc);
                acc = 1;
            }
        }
        mma_commit(bar_d + 8 * s);
    };

    /* the K padding columns (harmonics past nharms) of both A buffers stay zero */
    if (grp == 0) {
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const uint32_t ab = tmem + tlane + (uint32_t)(TM_A + KPAD * b);
#pragma unroll
            for (int c = NH; c < AHALF; c += 4) {
                tmem_st4(ab + c, 0, 0, 0, 0);
                tmem_st4(ab + AHALF + c, 0, 0, 0, 0);
            }
        }
    }
    /* prologue: tiles 0 and 1 */
    for (int i = 0; i < 2 && i < ntl; i++) {
        float2 xv[JB][4];
        load_x(i, xv);
        store_a(i, xv);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    int issued = 0;
    if (tid == 0)
        for (int i = 0; i < 2 && i < ntl; i++) issue(i);
    issued = min(2, ntl);
    bool ok = true;
    for (int it = 0; it < ntl; it++) {
        const int s = it & 1;
        float2 xv[JB][4];
        const bool next = it + 2 < ntl;
        if (next) load_x(it + 2, xv);
        const bool got = mbar_wait(bar_d + 8 * s, (it >> 1) & 1);
        if (__syncthreads_or(!got)) {
            if (tid == 0) atomicExch(a.err, 1);
            ok = false;
            break;
        }
        tc_fence_after();
        {
            const int tile = tile_begin + it;
            const int ci = a.tiles[3 * tile], j0 = a.tiles[3 * tile + 1];
            const int cnt = a.tiles[3 * tile + 2];
            const CsChunk &ch = a.chunks[ci];
            const uint32_t trow = tmem + (uint32_t)(TM_D + s * D_STRIDE) + tlane;
            C::epilogue4(grp, trow, ch, a, r < cnt, ci, j0 + r, lane, inv_scale);
        }
        if (next) store_a(s, xv);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (next && tid == 0) issue(s);
        if (next) issued++;
    }
    /* never free tensor memory under a transform in flight */
    if (!ok && tid == 0)
        for (int k = issued > 2 ? issued - 2 : 0; k < issued; k++)
            mbar_wait(bar_d + 8 * (k & 1), (k >> 1) & 1);
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

template <class C>
__global__ void __launch_bounds__(512, 1) search_pre(const __grid_constant__ Args a)
{
    pre_body<C>(a);
}

/* The same kernel over the tiles of several spectra (search_ws_multi). */
template <class C>
__global__ void __launch_bounds__(nthreads<C>(), 1)
search_ws_multi(const __grid_constant__ Args a0, const __grid_constant__ Multi mu)
{
    ws_body<C, true>(a0, mu);
}

}  // namespace wsk
