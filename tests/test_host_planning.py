"""Host planning of the B200 build against the reference, bit for bit (CPU).

The GPU kernel consumes host-built tables (trial grid, interpolation
weights and phase factors, chunk table, width banks, noise scales) and the
host collapses and formats candidates; all of it must equal the reference's.
Runs against libcoherent_search.so and oracle/_ref/libcsref.so.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200.search import Options

pytestmark = pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")

OURS = None


def ours():
    global OURS
    if OURS is None:
        OURS = nt.host_lib()
    return OURS


def params(lib, **kw):
    return Options(**kw).params(lib)


def plan_arrays(plans):
    out = []
    for i in range(plans.n):
        d = plans.plans[i]
        P, q, m = d.P, d.q, d.m
        rec = dict(h=d.h, m=m, q=q, s=d.s, base_adv=d.base_adv, pnum=d.pnum,
                   rfloor0=d.rfloor0, dr0=d.dr0, P=P)
        if P > 0:
            rec["row"] = np.ctypeslib.as_array(d.row, shape=(q,)).copy()
            rec["W"] = np.ctypeslib.as_array(d.W, shape=(m * P,)).copy()
            rec["A_re"] = np.ctypeslib.as_array(d.A_re, shape=(P,)).copy()
            rec["A_im"] = np.ctypeslib.as_array(d.A_im, shape=(P,)).copy()
            rec["carry"] = np.ctypeslib.as_array(d.carry, shape=(P,)).copy()
        out.append(rec)
    return out


@pytest.mark.parametrize("nharms,hidr,m,r_lo", [(60, 0.5, 16, 53.6870912), (32, 0.5, 16, 100.0),
                                                 (16, 0.25, 8, 7.3), (7, 0.5, 16, 1234.567),
                                                 (60, 0.5, 32, 0.0), (48, 1.0, 16, 12.5),
                                                 (60, 0.37, 16, 10.0)])
def test_direct_plans_identical(nharms, hidr, m, r_lo):
    res = []
    for lib in (ours(), rb.ref_lib()):
        p = params(lib, nharms=nharms, hidr=hidr, m=m)
        plans = nt.DirectPlanSet()
        assert lib.direct_plans_build(C.byref(plans), C.byref(p), r_lo) == 0
        res.append(plan_arrays(plans))
        lib.direct_plans_free(C.byref(plans))
    a, b = res
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.keys() == y.keys()
        for k in x:
            if isinstance(x[k], np.ndarray):
                np.testing.assert_array_equal(x[k], y[k], err_msg=k)
            else:
                assert x[k] == y[k], k


@pytest.mark.parametrize("lodr", [0.5 / 60, 0.5 / 32, 1 / 7, 0.25 / 16, 0.37 / 60, 0.1, 1e-6,
                                  3.0 / 65537])
def test_trial_grid_rational_identical(lodr):
    outs = []
    for lib in (ours(), rb.ref_lib()):
        pn, q = C.c_int(0), C.c_int(0)
        ok = lib.trial_grid_rational(lodr, C.byref(pn), C.byref(q))
        outs.append((ok, pn.value if ok else 0, q.value if ok else 0))
    assert outs[0] == outs[1]


@pytest.mark.parametrize("N,dt,nharms,blocksize,lofreq,hifreq,lobin",
                         [(1 << 20, 64e-6, 60, 2048, 0.1, 125.0, 100),
                          (1 << 16, 64e-6, 60, 65536, 0.1, 125.0, 100),
                          (1 << 16, 64e-6, 32, 1000, 0.1, 1000.0, 100),
                          (3 * 5 * 7 * 1024, 128e-6, 16, 777, 1.0, 3900.0, 100),
                          (1 << 14, 64e-6, 60, 512, 0.1, 125.0, 8)])
def test_chunk_starts_identical(N, dt, nharms, blocksize, lofreq, hifreq, lobin):
    amps = np.zeros(N, dtype=np.float32)          # N/2 complex
    opts = Options(nharms=nharms, blocksize=blocksize, lofreq=lofreq, hifreq=hifreq, lobin=lobin)
    r_lo, lodr, total = opts.geometry(N, dt)
    got = []
    for lib in (ours(), rb.ref_lib()):
        ft = rb.make_file(amps, N, dt)
        p = opts.params(lib)
        plans = nt.DirectPlanSet()
        assert lib.direct_plans_build(C.byref(plans), C.byref(p), r_lo) == 0
        cs = C.POINTER(C.c_longlong)()
        n = C.c_longlong(0)
        assert lib.chunk_starts(C.byref(plans), C.byref(ft), C.byref(p), total, blocksize,
                                C.byref(cs), C.byref(n)) == 0
        got.append(np.ctypeslib.as_array(cs, shape=(n.value,)).copy())
        C.CDLL(None).free(cs)
        fits = [lib.cs_harmonic_fits(C.byref(plans.plans[h]), C.byref(ft), C.byref(p), t)
                for h in range(nharms) for t in (0, total // 3, total - 1)]
        got.append(np.array(fits))
        lib.direct_plans_free(C.byref(plans))
    np.testing.assert_array_equal(got[0], got[2])
    np.testing.assert_array_equal(got[1], got[3])


@pytest.mark.parametrize("maxdecim", [1, 2, 6, 8, 16])
@pytest.mark.parametrize("nharms", [8, 16, 32, 60, 64])
def test_widths_sigma_shape_identical(maxdecim, nharms):
    rng = np.random.default_rng(nharms * 100 + maxdecim)
    for lib_pair in [(ours(), rb.ref_lib())]:
        pa = Options(nharms=nharms, maxdecim=maxdecim).params(lib_pair[0])
        pb = Options(nharms=nharms, maxdecim=maxdecim).params(lib_pair[1])
        for k in list(pa.decimations)[:pa.ndecim]:
            Hk = nharms // k
            nb = 2 * Hk
            wa = (C.c_int * 256)()
            wb = (C.c_int * 256)()
            na = lib_pair[0].ladder_boxcar_widths(nb, k, C.byref(pa), wa, 256)
            nbw = lib_pair[1].ladder_boxcar_widths(nb, k, C.byref(pb), wb, 256)
            assert na == nbw and list(wa)[:na] == list(wb)[:nbw]
            for trial in range(6):
                filled = (rng.random(nharms) < (0.5 if trial else 1.1)).astype(np.uint8)
                fp = filled.ctypes.data_as(C.POINTER(C.c_uint8))
                sa = lib_pair[0].analytic_sigma(fp, k, Hk)
                sb = lib_pair[1].analytic_sigma(fp, k, Hk)
                assert sa == sb
                sha = (C.c_double * 256)()
                shb = (C.c_double * 256)()
                lib_pair[0].boxcar_shape(sha, nb, wa, na, fp, k, Hk)
                lib_pair[1].boxcar_shape(shb, nb, wb, nbw, fp, k, Hk)
                assert list(sha)[:na] == list(shb)[:na]


def _random_cands(rng, n):
    r = np.sort(rng.uniform(50, 5000, n))
    near = rng.random(n) < 0.3
    r[near] += rng.uniform(0, 2, size=near.sum())
    harm = rng.random(n) < 0.2
    r[harm] = r[rng.integers(0, n, harm.sum())] * rng.integers(2, 5, harm.sum())
    arr = np.zeros(n, dtype=nt.CAND_DTYPE)
    arr["r"] = r
    arr["freq"] = r / 536.870912
    arr["metric"] = np.round(rng.uniform(8, 40, n), 2)   # ties on purpose
    arr["nharm"] = rng.choice([60, 30, 20, 15, 12, 10], n)
    arr["ducy"] = np.nan
    return arr


def _as_list(arr):
    buf = (nt.Candidate * max(arr.size, 1))()
    C.memmove(buf, arr.ctypes.data, arr.size * C.sizeof(nt.Candidate))
    return buf, nt.CandidateList(C.cast(buf, C.POINTER(nt.Candidate)), arr.size, arr.size)


@pytest.mark.parametrize("seed", range(5))
def test_collapse_identical(seed):
    rng = np.random.default_rng(seed)
    arr = _random_cands(rng, 400)
    res = []
    for lib in (ours(), rb.ref_lib()):
        _, cl = _as_list(arr)
        d = lib.remove_duplicates(C.byref(cl), 1.0)
        h = lib.remove_harmonics(C.byref(d), 16, 1.0)
        res.append((nt.candidates_to_numpy(d), nt.candidates_to_numpy(h)))
    for x, y in zip(res[0], res[1]):
        assert x.size == y.size
        for f in ("freq", "metric", "r", "nharm"):
            np.testing.assert_array_equal(x[f], y[f], err_msg=f)


def test_cohout_text_identical():
    rng = np.random.default_rng(7)
    arr = _random_cands(rng, 50)
    arr["ducy"][::3] = rng.uniform(0.01, 0.3, len(arr["ducy"][::3]))
    texts = []
    with tempfile.TemporaryDirectory() as d:
        for i, lib in enumerate((ours(), rb.ref_lib())):
            _, cl = _as_list(arr)
            path = os.path.join(d, f"{i}.cohout").encode()
            assert lib.write_candidates(C.byref(cl), path, 8.0) == 0
            texts.append(open(path, "rb").read())
    assert texts[0] == texts[1]


def test_measure_ducy_matches_reference():
    """Duty cycles from the m=64 FP64 candidate profile (direct c2r here,
    FFTW-shim c2r in the reference): same best width."""
    import glob
    z = np.load(sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "small60.npz")))[0])
    raw = z["raw"][:40]
    amps = z["amps"]
    N, dt = int(z["N"]), float(z["dt"])
    out = []
    for lib in (ours(), rb.ref_lib()):
        ft = rb.make_file(amps, N, dt)
        p = Options().params(lib)
        _, cl = _as_list(raw)
        res = lib.measure_ducy(C.byref(ft), C.byref(cl), C.byref(p))
        out.append(nt.candidates_to_numpy(res)["ducy"])
    np.testing.assert_array_equal(out[0], out[1])


def test_search_file_refuses_cpu_path():
    lib = ours()
    amps = np.zeros(1 << 12, dtype=np.float32)
    ft = rb.make_file(amps, 1 << 12, 64e-6)
    p = Options().params(lib)
    cl = lib.search_file(C.byref(ft), C.byref(p), 0.1, 125.0, 100, 0, 8.0, 1, 1.0, 1, 16, None,
                         0, 0, 0, None, None, 1.0, -1)
    assert cl.n == 0
