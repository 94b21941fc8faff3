"""The oracle is pinned before it is trusted (CPU only).

* the FFTW-API shim against numpy's FFT (the transform the reference calls);
* oracle/cs_oracle.c against the golden fixtures made from the reference
  (tests/golden/make_golden.py) and, when the reference library is built,
  against the reference run live on a fresh seeded input.
Candidate identity (r, harmonic count, order) is exact; S/N agrees to 1e-5
relative (the oracle's c2r is evaluated in FP64, the reference's in FP32).
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
SNR_RTOL = 1e-5

needs_ref = pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")


def load_case(path):
    z = np.load(path, allow_pickle=False)
    o = {k[4:]: z[k].item() for k in z.files if k.startswith("opt_")}
    return z, Options(**o)


def compare_raw(got, want, rtol=SNR_RTOL):
    assert got.size == want.size
    np.testing.assert_array_equal(got["r"], want["r"])
    np.testing.assert_array_equal(got["nharm"], want["nharm"])
    np.testing.assert_allclose(got["metric"], want["metric"], rtol=rtol)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden(path):
    z, opts = load_case(path)
    N, dt = int(z["N"]), float(z["dt"])
    total = int(z["total"])
    met, geo = rb.oracle_metrics(z["amps"], N, dt, opts, 0, total)
    ora = rb.oracle_candidates(met, geo, N, dt, opts)
    ora = ora[np.argsort(ora["freq"], kind="stable")]
    compare_raw(ora, z["raw"])
    # FP64 mode against the reference's --precision f64 path
    met64, _ = rb.oracle_metrics(z["amps"], N, dt, opts, 0, total, prec64=True)
    ora64 = rb.oracle_candidates(met64, geo, N, dt, opts)
    ora64 = ora64[np.argsort(ora64["freq"], kind="stable")]
    compare_raw(ora64, z["raw64"], rtol=1e-9)


@needs_ref
def test_oracle_matches_reference_live():
    spec = synth.SeriesSpec(N=1 << 15, dt=64e-6, seed=909, pulsars=[synth.Pulsar(63.1, 0.03, 30.0)],
                            red_index=-2.0, red_amp=0.3)
    x = synth.make_series(spec)
    amps = rb.ref_spectrum(x, spec.dt)
    opts = Options(blocksize=1000, threshold=5.0)     # chunk edges off the tile grid
    ref = rb.ref_search(amps, spec.N, spec.dt, opts, collapse=False)
    _, _, total, _ = rb.ref_chunks(amps, spec.N, spec.dt, opts)
    met, geo = rb.oracle_metrics(amps, spec.N, spec.dt, opts, 0, total)
    ora = rb.oracle_candidates(met, geo, spec.N, spec.dt, opts)
    compare_raw(ora[np.argsort(ora["freq"], kind="stable")], ref)


def _dedispersed_spectrum(dm: int):
    """A dedispersed, padded series of the 256-channel front-end case: 24576
    points at 128 us, so the top harmonics pass Nyquist over most of the band
    and chunks carry partial harmonic sets at both ends."""
    from coherentsearch_c_b200.prep import running_mean
    from test_dedisp import GEOMS, fb_for, ours_tables
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=40, seed=11)
    numout = 24576
    out = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                            t.blocks_per_read, numout)
    pad = np.float32(running_mean(out[0]))
    series = np.concatenate([out[dm], np.full(numout - out.shape[1], pad, np.float32)])
    return rb.ref_spectrum(series, g[7]), numout, g[7]


needs_dedisp_ref = pytest.mark.skipif(not (rb.have_ref() and rb.have_dedisp_ref()),
                                      reason="oracle/_ref not built")


@needs_dedisp_ref
def test_oracle_matches_reference_partial_harmonics():
    amps, N, dt = _dedispersed_spectrum(25)
    opts = Options(blocksize=4096, threshold=6.0)
    ref = rb.ref_search(amps, N, dt, opts, collapse=False)
    _, _, total, _ = rb.ref_chunks(amps, N, dt, opts)
    met, geo = rb.oracle_metrics(amps, N, dt, opts, 0, total)
    ora = rb.oracle_candidates(met, geo, N, dt, opts)
    compare_raw(ora[np.argsort(ora["freq"], kind="stable")], ref)


@needs_dedisp_ref
def test_reference_threads_change_its_result():
    """Why the checkers pin the reference to one thread: on 16 threads its
    per-workspace boxcar-shape cache goes stale in one chunk (trials
    25815..26276, thread 0's successor of chunk 16) and it reports extra
    decimated-slot candidates there, all of them outside the one-thread set."""
    amps, N, dt = _dedispersed_spectrum(25)
    opts = Options(blocksize=4096, threshold=6.0)
    one = rb.ref_search(amps, N, dt, opts, collapse=False)
    try:
        rb.pin_ref_threads(16)
        many = rb.ref_search(amps, N, dt, opts, collapse=False)
    finally:
        rb.pin_ref_threads(1)
    r_lo, lodr, _, cstarts = rb.ref_chunks(amps, N, dt, opts)
    c = int(np.searchsorted(cstarts, 25815))
    assert cstarts[c] == 25815 and c % 16 == (c - 16) % 16
    key = lambda a: set(zip(np.round(a["r"], 9), a["nharm"]))
    extra = key(many) - key(one)
    assert many.size > one.size and len(extra) == many.size - one.size
    for r, h in extra:
        k = opts.nharms // int(h)
        assert k > 1
        trial = (r / k - r_lo) / lodr
        assert cstarts[c] - 0.5 <= trial < cstarts[c + 1] - 0.5


@needs_ref
def test_golden_reference_reproducible():
    """The fixtures are what the reference produces here today."""
    z, opts = load_case(GOLDEN[0])
    N, dt = int(z["N"]), float(z["dt"])
    raw = rb.ref_search(z["amps"], N, dt, opts, collapse=False)
    compare_raw(raw, z["raw"], rtol=0)


@needs_ref
def test_golden_spectrum_pipeline():
    """realfft + rednoise of the stored series reproduces the stored spectrum."""
    path = [p for p in GOLDEN if "series" in np.load(p).files][0]
    z, _ = load_case(path)
    amps = rb.ref_spectrum(z["series"], float(z["dt"]))
    np.testing.assert_array_equal(amps, z["amps"])


@needs_ref
@pytest.mark.parametrize("n", [4, 10, 24, 40, 64, 120, 2 * 97])
def test_shim_c2r_matches_numpy(n):
    lib = rb.ref_lib()
    lib.fftwf_plan_many_dft_c2r.restype = C.c_void_p
    lib.fftwf_execute.argtypes = [C.c_void_p]
    lib.fftwf_destroy_plan.argtypes = [C.c_void_p]
    rng = np.random.default_rng(n)
    N, B = n // 2, 40
    X = (rng.standard_normal((N + 1, B)) + 1j * rng.standard_normal((N + 1, B))).astype(np.complex64)
    out = np.zeros((B, n), np.float32)
    nn = (C.c_int * 1)(n)
    p = lib.fftwf_plan_many_dft_c2r(1, nn, B, X.ctypes.data_as(C.c_void_p), None, B, 1,
                                    out.ctypes.data_as(C.c_void_p), None, 1, n, 0)
    lib.fftwf_execute(C.c_void_p(p))
    lib.fftwf_destroy_plan(C.c_void_p(p))
    Xd = X.astype(np.complex128).T
    full = np.concatenate([Xd[:, :1].real, Xd[:, 1:N], Xd[:, N:N + 1].real], axis=1)
    ref = np.fft.irfft(full, n=n, axis=1) * n
    assert np.abs(out - ref).max() <= 3e-6 * np.abs(ref).max()


@needs_ref
@pytest.mark.parametrize("n", [60, 4096, 3 * 5 * 7 * 11, 2 * 104729])
def test_shim_complex_forward_matches_numpy(n):
    lib = rb.ref_lib()
    lib.fftwf_plan_dft_1d.restype = C.c_void_p
    lib.fftwf_execute.argtypes = [C.c_void_p]
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    y = np.zeros(n, np.complex64)
    p = lib.fftwf_plan_dft_1d(n, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), -1, 64)
    lib.fftwf_execute(C.c_void_p(p))
    ref = np.fft.fft(x.astype(np.complex128))
    assert np.abs(y - ref).max() <= 5e-6 * np.abs(ref).max()
