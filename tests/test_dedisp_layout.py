"""The integer DM stage's tables and index arithmetic, restated on the CPU.

dd_dms_u16 (cs_dedisp.cu) reads S in words that hold two samples, w and
w + DM_P, and stages per (tile, group of G DMs) one window per subband with
bulk copies.  This test restates cs_dedisp_create's tables (window starts,
shared words, codes, stage layout, row stride) and the kernel's reads, and
checks for the dedispersion geometries under test and the bench workload:

  * every bulk copy starts and ends on a 16-byte boundary, inside S's rows;
  * every (DM, subband) row of DM_P words a summing thread reads lies inside
    its subband's window in the stage; padding reads the zero row;
  * the stages fit in shared memory and every code fits 16 bits;
  * an emulation of the staged sums equals the direct formula
    out_d[T] = sum_s S_s[T + off_ds], bit for bit (integers).
"""
import numpy as np
import pytest

from coherentsearch_c_b200.dedisp import dedisp_tables

P, TILE, GMAX, MAXST = 128, 256, 32, 4
OPTIN = 232448                                  # B200 shared memory per CTA (opt-in)

FB_LO, FB_CW = 1400.0 + 0.5 * 300.0 / 1024 - 150.0, 300.0 / 1024
GEOMS = {
    "bench_1024x64x500": ((1024, 64, 500, 0.0, 0.4, FB_LO, FB_CW, 64e-6, 2400), 1 << 22),
    "filterbank_1024x64x500": ((1024, 64, 500, 0.0, 0.4, FB_LO, FB_CW, 64e-6, 2400), 12 * 2400),
    "c256_s16_d40": ((256, 16, 40, 10.0, 1.5, 1200.0, 1.0, 128e-6, 600), 11 * 600 + 200),
    "c200_s8_d25_cps25": ((200, 8, 25, 0.0, 3.0, 400.0, 0.5, 256e-6, 1200), 10 * 1200 + 400),
    "c64_s64_d7": ((64, 64, 7, 0.0, 20.0, 800.0, 0.5, 64e-6, 800), 14 * 800 + 266),
    # offsets of ~70,000 samples: groups of one DM
    "wide": ((64, 64, 7, 100.0, 25.0, 150.0, 0.125, 64e-6, 800), 100 * 800),
}


def plan(offs, max_spectra):
    """cs_dedisp_create's DM-stage tables."""
    ndm, nsub = offs.shape
    nsub8 = (nsub + 7) // 8 * 8
    G = GMAX
    while G >= 1:
        ng = (ndm + G - 1) // G
        win = np.zeros((ng, nsub, 3), np.int64)
        wmax = 0
        for g in range(ng):
            o = offs[g * G:(g + 1) * G]
            wb = 0
            for s in range(nsub):
                start = int(o[:, s].min()) & ~3
                words = (int(o[:, s].max()) - start + P + 3) // 4 * 4
                win[g, s] = (start, wb, words)
                wb += words
            wmax = max(wmax, wb)
        code_bytes = 2 * G * nsub8
        code_word = wmax
        zero_word = wmax + code_bytes // 4
        stage_words = (zero_word + P + 31) // 32 * 32
        nstage = min(MAXST, (OPTIN - 1024) // (4 * stage_words))
        if nstage >= 2 and zero_word < 65536:
            break
        G //= 2
    if G < 1:
        return None
    code = np.full((ng, G, nsub8), zero_word, np.int64)
    for g in range(ng):
        for dl in range(G):
            d = g * G + dl
            if d >= ndm:
                continue
            code[g, dl, :nsub] = win[g, :, 1] + offs[d] - win[g, :, 0]
    ntile = (max_spectra + TILE - 1) // TILE
    sstride = ((ntile + 1) * TILE + int(offs.max()) + 64 + 255) // 256 * 256
    return dict(G=G, ng=ng, win=win, code=code, code_word=code_word, zero_word=zero_word,
                stage_words=stage_words, nstage=nstage, sstride=sstride, nsub8=nsub8,
                code_bytes=code_bytes)


def _tables(name):
    g, max_spectra = GEOMS[name]
    t = dedisp_tables(*g[:8], g[8])
    return t, max_spectra


@pytest.mark.parametrize("name", list(GEOMS))
def test_stage_layout_in_bounds(name):
    t, max_spectra = _tables(name)
    offs = t.offsets.astype(np.int64)
    pl = plan(offs, max_spectra)
    assert pl is not None
    win, code = pl["win"], pl["code"]
    assert pl["nstage"] * pl["stage_words"] * 4 <= OPTIN - 1024
    assert pl["zero_word"] + P <= pl["stage_words"] and pl["zero_word"] < 65536
    assert pl["code_word"] % 4 == 0 and pl["code_bytes"] % 16 == 0
    assert pl["stage_words"] % 4 == 0 and pl["sstride"] % 4 == 0
    # windows: 16-byte aligned in S and in the stage, inside the window area
    assert np.all(win[..., 0] % 4 == 0) and np.all(win[..., 1] % 4 == 0)
    assert np.all(win[..., 2] % 4 == 0)
    assert np.all(win[..., 1] + win[..., 2] <= pl["code_word"])
    # the furthest copy of the last tile stays inside its row
    ntile = (max_spectra + TILE - 1) // TILE
    T0 = (ntile - 1) * TILE
    assert np.all(T0 + win[..., 0] + win[..., 2] <= pl["sstride"])
    # every DM row inside its subband's window (or the zero row)
    ndm, nsub = offs.shape
    for g in range(pl["ng"]):
        for dl in range(pl["G"]):
            c = code[g, dl]
            if g * pl["G"] + dl >= ndm:
                assert np.all(c == pl["zero_word"])
                continue
            assert np.all(c[:nsub] >= win[g, :, 1])
            assert np.all(c[:nsub] + P <= win[g, :, 1] + win[g, :, 2])
            assert np.all(c[nsub:] == pl["zero_word"])


@pytest.mark.parametrize("name", ["c256_s16_d40", "c200_s8_d25_cps25", "c64_s64_d7"])
def test_staged_sums_equal_formula(name):
    t, max_spectra = _tables(name)
    offs = t.offsets.astype(np.int64)
    ndm, nsub = offs.shape
    pl = plan(offs, max_spectra)
    sstride = pl["sstride"]
    rng = np.random.default_rng(3)
    S = rng.integers(0, 4000, size=(nsub, sstride), dtype=np.int64)
    # S' words: low half sample w, high half sample w + P
    Sw = S.copy()
    Sw[:, :-P] |= S[:, P:] << 16
    nout = max_spectra - int(offs.max()) - 1
    ntile = (nout + TILE - 1) // TILE
    out = np.zeros((ndm, ntile * TILE), np.int64)
    G = pl["G"]
    for tile in range(ntile):
        T0 = tile * TILE
        for g in range(pl["ng"]):
            stage = np.zeros(pl["stage_words"], np.int64)
            for s in range(nsub):
                start, wb, words = pl["win"][g, s]
                stage[wb:wb + words] = Sw[s, T0 + start:T0 + start + words]
            for dl in range(G):
                d = g * G + dl
                if d >= ndm:
                    continue
                lo = np.zeros(P, np.int64)
                hi = np.zeros(P, np.int64)
                for s in range(pl["nsub8"]):
                    w = stage[pl["code"][g, dl, s] + np.arange(P)]
                    lo += w & 0xffff
                    hi += w >> 16
                out[d, T0:T0 + P] = lo
                out[d, T0 + P:T0 + TILE] = hi
    ref = np.zeros((ndm, nout), np.int64)
    for d in range(ndm):
        for s in range(nsub):
            ref[d] += S[s, offs[d, s]:offs[d, s] + nout]
    np.testing.assert_array_equal(out[:, :nout], ref)


FD_T = 256


def fplan(offs, max_spectra):
    """cs_dedisp_create's tables of the clipped (float) DM stage."""
    ndm, nsub = offs.shape
    nsub8 = (nsub + 7) // 8 * 8
    G = GMAX
    while G >= 1:
        ng = (ndm + G - 1) // G
        win = np.zeros((ng, nsub, 3), np.int64)
        wmax = 0
        for g in range(ng):
            o = offs[g * G:(g + 1) * G]
            wb = 0
            for s in range(nsub):
                start = int(o[:, s].min()) & ~3
                n = (int(o[:, s].max()) - start + FD_T + 3) // 4 * 4
                win[g, s] = (start, wb, n)
                wb += n
            wmax = max(wmax, wb)
        code_bytes = 2 * G * nsub8
        stage_words = (wmax + code_bytes // 4 + 31) // 32 * 32
        nstage = min(MAXST, (OPTIN - 1024) // (4 * stage_words))
        if nstage >= 2 and wmax < 65536:
            return dict(G=G, ng=ng, win=win, code_word=wmax, code_bytes=code_bytes,
                        stage_words=stage_words, nstage=nstage, nsub8=nsub8)
        G //= 2
    return None


@pytest.mark.parametrize("name", list(GEOMS))
def test_float_stage_layout_in_bounds(name):
    t, max_spectra = _tables(name)
    offs = t.offsets.astype(np.int64)
    ndm, nsub = offs.shape
    pl = fplan(offs, max_spectra)
    assert pl is not None
    win = pl["win"]
    assert pl["nstage"] * pl["stage_words"] * 4 <= OPTIN - 1024
    assert pl["code_word"] % 4 == 0 and pl["code_bytes"] % 16 == 0
    assert pl["code_word"] + pl["code_bytes"] // 4 <= pl["stage_words"]
    assert np.all(win[..., 0] % 4 == 0) and np.all(win[..., 1] % 4 == 0)
    assert np.all(win[..., 2] % 4 == 0)
    assert np.all(win[..., 1] + win[..., 2] <= pl["code_word"])
    ntile = (max_spectra + TILE - 1) // TILE
    sstride = ((ntile + 1) * TILE + int(offs.max()) + 64 + 255) // 256 * 256
    T0 = (ntile - 1) * FD_T
    assert np.all(T0 + win[..., 0] + win[..., 2] <= sstride)
    G = pl["G"]
    for g in range(pl["ng"]):
        for dl in range(G):
            d = g * G + dl
            if d >= ndm:
                continue
            c = win[g, :, 1] + offs[d] - win[g, :, 0]
            assert np.all(c >= win[g, :, 1]) and np.all(c + FD_T <= win[g, :, 1] + win[g, :, 2])
            assert np.all(c < 65536)
