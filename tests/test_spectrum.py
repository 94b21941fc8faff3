"""Time series -> spectrum on the GPU (cs_spectrum_*) against the
reference's datpipe realfft + rednoise (oracle/_ref/libcsref.so).

The reference's FFT (FFTW through the shim, then a double-precision split
with recurrent twiddles) fixes its last bits; any other FFT differs there.
Tolerances: every normalised bin within 2e-5 of the reference's, absolute
(bins are O(1) after normalisation); bin 0 exactly (1, 0); and the search of
the GPU spectrum finds the reference's candidates under the search parity
tolerances (tests/test_gpu_parity.py)."""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session
from coherentsearch_c_b200.spectrum import SpectrumMaker

from test_gpu_parity import SNR_RTOL_F32, match_candidates

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")]

BIN_ATOL = 2e-5
DT = 64e-6


def series(N, seed, red=False):
    spec = synth.SeriesSpec(N=N, dt=DT, seed=seed, pulsars=[synth.Pulsar(13.1, 0.05, 30.0)],
                            red_index=-2.0 if red else None, red_amp=0.3 if red else 0.0)
    return synth.make_series(spec)


@pytest.mark.parametrize("N,red", [(1 << 15, False), (3 * (1 << 14), True), (1 << 18, True),
                                   (1000 * 1024, False)])
def test_spectrum_matches_reference(gpu_ready, N, red):
    x = series(N, seed=N % 997, red=red)
    ref = rb.ref_spectrum(x, DT)
    with SpectrumMaker(N, DT) as sm:
        got = sm.run(x)
        again = sm.run(x)
    np.testing.assert_array_equal(got, again)          # a plan is reusable
    assert got[0] == 1.0 and got[1] == 0.0
    err = np.abs(got - ref)
    assert err.max() <= BIN_ATOL, (err.max(), int(err.argmax()))


def test_search_of_gpu_spectrum(gpu_ready):
    N = 1 << 17
    x = series(N, seed=42, red=True)
    opts = Options(blocksize=4096, threshold=6.0)
    ref = rb.ref_search(rb.ref_spectrum(x, DT), N, DT, opts, collapse=False)
    with SpectrumMaker(N, DT) as sm:
        amps = sm.run(x)
    ses = Session(N, DT, opts)
    try:
        got = ses.run_raw(amps)
    finally:
        ses.close()
    got = got[np.argsort(got["freq"], kind="stable")]
    match_candidates(got, ref, opts.threshold, SNR_RTOL_F32)
