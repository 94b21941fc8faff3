/*
 * The FP64 search (--precision f64, the reference's CS_PREC_F64): the same
 * trials, chunks and records as the FP32 kernels, with the profile stage in
 * double precision as the reference computes it (src/cuda.cu:579-584, 621,
 * 726, 1004-1014 on its GPU; src/search.c:288-292, 333-400, 641-656 and
 * src/boxcar.c:203-252, 715-731 on its CPU):
 *
 *   1. interpolation in FP32, bit-identical to the FP32 kernels, the
 *      amplitude then widened to double (src/interp.c:555-573: "the products
 *      are formed in f32 and widened per element");
 *   2. the unnormalised c2r of each profile-producing slot (the base profile
 *      and every decimation that does not fold) in FP64.  The reference runs
 *      FFTW / cuFFT Z2D; here it is a dense half-spectrum DFT: for bin
 *      n = 0..Hk the cosine part C_n = sum_h Re X_h c_hn and the sine part
 *      S_n = sum_h Im X_h s_hn, so x[n] = C_n - S_n and x[2Hk-n] = C_n + S_n
 *      (cs_tables_dft_f64).  Each thread accumulates 4 trials x 2 bins of
 *      both parts with DFMA from shared memory;
 *   3. the k-fold averages (fold_row_f64: left-to-right sum, times 1/k), the
 *      cyclic prefix sums and the exact boxcar scan (profile_boxcar_f64) in
 *      double with the reference's expression order, one warp per slot and
 *      one lane per trial; the scan is the exact one the reference's f64 gate
 *      falls back to for every trial that can reach the threshold;
 *   4. threshold in double and warp-ballot compaction into CsRec64 records.
 *
 * Work unit: 32 trials (a quarter of a 128-trial tile).  One CTA of 256
 * threads per SM, persistent over the sub-tiles.
 *
 * Shared memory: the DFT tables (cos then sin, nh x ucols doubles each), the
 * profile rows (32 x prs doubles, prs odd so lanes on consecutive trials hit
 * different banks) and the prefix-sum arrays of every slot (pos-major, 32
 * trials a row).  The FP32 amplitudes of step 1 live in the prefix-sum
 * region, which is free until step 3.
 */
#pragma once

namespace f64k {

constexpr int TT = 32;              /* trials per sub-tile */
constexpr int NT = 256;             /* threads per CTA */

struct Extra {
    const double *bcs;              /* cos table [nh][ucols], then sin table */
    int nunit, ucols;
    int unit0[CS_MAX_SLOT];         /* first DFT unit of a profile slot, or -1 */
    int prs;                        /* profile row stride (doubles, odd) */
    int ps_off[CS_MAX_SLOT];        /* prefix-sum array of each slot (doubles) */
    int ps_total;                   /* doubles in all prefix-sum arrays */
    const double *scales;           /* per chunk CS_F64_SCALES */
    CsRec64 *recs;
};

/* Shared-memory bytes of the kernel for a table layout. */
static __host__ __device__ inline int smem_bytes(int nh, int ucols, int prs, int ps_total)
{
    return 2 * nh * ucols * 8 + TT * prs * 8 + ps_total * 8;
}

/* x[j] of a slot's profile for one trial: its own DFT columns, or the k-fold
 * average of the base profile (src/search.c:333-365: a = s[j], a += s[j +
 * q*nk] for q = 1..k-1, times 1/k). */
static __device__ __forceinline__ double slot_value(const double *row, const CsSlot &sl,
                                                    double invk, int j)
{
    if (!sl.fold) return row[sl.col0 + j];
    double a = row[j];
    for (int q = 1; q < sl.k; q++) a = __dadd_rn(a, row[j + q * sl.nk]);
    return __dmul_rn(a, invk);
}

template <int MT>
__global__ void __launch_bounds__(NT, 1)
search_f64(const SearchArgs args, const Extra ex)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ CsHarm harm_s[CS_MAX_NH];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nh = args.nh, ucols = ex.ucols, prs = ex.prs;
    const int m = MT ? MT : args.m;
    double *bc = reinterpret_cast<double *>(smem);
    double *bs = bc + (size_t)nh * ucols;
    double *pr = bs + (size_t)nh * ucols;
    double *ps = pr + (size_t)TT * prs;
    float *xr = reinterpret_cast<float *>(ps);       /* [nh][TT], then xi */
    float *xi = xr + (size_t)nh * TT;

    for (int h = tid; h < nh; h += NT) harm_s[h] = args.harm[h];
    for (int i = tid; i < 2 * nh * ucols; i += NT) bc[i] = ex.bcs[i];
    __syncthreads();

    const int nsub = args.ntiles * (CS_TILE_M / TT);
    for (int item = blockIdx.x; item < nsub; item += gridDim.x) {
        const int tile = item / (CS_TILE_M / TT), sub = item % (CS_TILE_M / TT);
        const int ci = args.tiles[3 * tile + 0];
        const int j0 = args.tiles[3 * tile + 1] + sub * TT;
        const int cnt = args.tiles[3 * tile + 2] - sub * TT;
        if (cnt <= 0) continue;                     /* uniform over the CTA */
        const CsChunk &ch = args.chunks[ci];

        /* ---- 1. FP32 interpolation: lane = trial, warp = harmonic phase ---- */
        {
            const int r = lane;
            const bool valid = r < cnt;
            const long long t = ch.i0 + j0 + r;
            const long long tp = t * (long long)args.pnum;
            const long long Q = tp / args.q;
            const uint32_t R = (uint32_t)(tp - Q * args.q);
            for (int h = warp + 1; h <= nh; h += NT / 32) {
                float2 x = make_float2(0.0f, 0.0f);
                if (valid && ((ch.filled >> (h - 1)) & 1ULL))
                    x = interp_amp<MT>(args, harm_s[h - 1], h, m, Q, R);
                xr[(h - 1) * TT + r] = x.x;
                xi[(h - 1) * TT + r] = x.y;
            }
        }
        __syncthreads();

        /* ---- 2. FP64 half-spectrum DFT: 4 trials x 2 units per item ---- */
        for (int w = tid; w < (TT / 4) * (ucols / 2); w += NT) {
            const int tg = w & (TT / 4 - 1), ug = w / (TT / 4);
            double c[4][2], s[4][2];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) c[i][j] = s[i][j] = 0.0;
            const float4 *xr4 = reinterpret_cast<const float4 *>(xr) + tg;
            const float4 *xi4 = reinterpret_cast<const float4 *>(xi) + tg;
            const double2 *bc2 = reinterpret_cast<const double2 *>(bc) + ug;
            const double2 *bs2 = reinterpret_cast<const double2 *>(bs) + ug;
            for (int h = 0; h < nh; h++) {
                const float4 a = xr4[h * (TT / 4)], b = xi4[h * (TT / 4)];
                const double2 cw = bc2[h * (ucols / 2)], sw = bs2[h * (ucols / 2)];
                const double ar[4] = {a.x, a.y, a.z, a.w}, ai[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    c[i][0] = __fma_rn(ar[i], cw.x, c[i][0]);
                    c[i][1] = __fma_rn(ar[i], cw.y, c[i][1]);
                    s[i][0] = __fma_rn(ai[i], sw.x, s[i][0]);
                    s[i][1] = __fma_rn(ai[i], sw.y, s[i][1]);
                }
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int u = 2 * ug + j;
                if (u >= ex.nunit) continue;
                int sl = 0;
                for (int q = 0; q < args.nslot; q++)
                    if (ex.unit0[q] >= 0 && u >= ex.unit0[q]) sl = q;
                const int n = u - ex.unit0[sl], Hk = args.slot[sl].Hk;
                const int col0 = args.slot[sl].col0;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    double *row = pr + (size_t)(4 * tg + i) * prs + col0;
                    row[n] = __dsub_rn(c[i][j], s[i][j]);
                    if (n > 0 && n < Hk) row[2 * Hk - n] = __dadd_rn(c[i][j], s[i][j]);
                }
            }
        }
        __syncthreads();

        /* ---- 3. folds, prefix sums, boxcar scan: warp = slot, lane = trial ---- */
        if (warp < args.nslot) {
            const CsSlot &sl = args.slot[warp];
            const int r = lane, nk = sl.nk;
            const double *row = pr + (size_t)r * prs;
            double *P = ps + ex.ps_off[warp];
            const double invk = 1.0 / (double)sl.k;
            /* psum[i] = psum[i-1] + x[(i-1) mod nk], i = 1..nk+wmax
             * (src/boxcar.c:203-211 with b = 0) */
            double acc = 0.0;
            P[r] = 0.0;
            for (int i = 1; i <= nk + sl.wmax; i++) {
                const int idx = i > nk ? i - nk : i;
                acc = __dadd_rn(acc, slot_value(row, sl, invk, idx - 1));
                P[i * TT + r] = acc;
            }
            const double *sc = ex.scales + (size_t)ci * CS_F64_SCALES + warp * (CS_NWMAX + 1);
            double best = -INFINITY;
            if (!(sc[0] > 0.0)) {
                best = 0.0;                     /* profile_boxcar_f64: no noise scale */
            } else {
                const double stot = __dsub_rn(P[nk * TT + r], P[r]);
                for (int a = 0; a < sl.nw; a++) {
                    const int w = sl.widths[a];
                    const double duty = __ddiv_rn((double)w, (double)nk);
                    double mx = __dsub_rn(P[w * TT + r], P[r]);
                    for (int p = 2; p <= nk; p++) {
                        const double d = __dsub_rn(P[(p + w - 1) * TT + r], P[(p - 1) * TT + r]);
                        if (d > mx) mx = d;
                    }
                    const double cand = __dmul_rn(__dsub_rn(mx, __dmul_rn(duty, stot)), sc[1 + a]);
                    if (cand > best) best = cand;
                }
            }
            /* ---- 4. threshold + warp-aggregated compaction ---- */
            const int j = j0 + r;
            const bool hit = r < cnt && j < ch.nvalid[warp] && best > args.thresh;
            const unsigned mask = __ballot_sync(0xffffffffu, hit);
            if (mask) {
                unsigned basei = 0;
                if (lane == 0) basei = atomicAdd(args.count, (unsigned)__popc(mask));
                basei = __shfl_sync(0xffffffffu, basei, 0);
                if (hit) {
                    const unsigned pos = basei + (unsigned)__popc(mask & ((1u << lane) - 1u));
                    if (pos < args.cap) {
                        CsRec64 rec;
                        rec.chunk = ci;
                        rec.slot = warp;
                        rec.j = j;
                        rec.pad = 0;
                        rec.metric = best;
                        ex.recs[pos] = rec;
                    }
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace f64k
