"""Duty cycles on the GPU (cs_ducy_*, Session.measure_ducy) against the host
measure_ducy restatement and the reference's own (src/candidate.c:305-329,
FFTW-shim c2r): the same best width for every candidate."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")]


def _host_ducy(lib, amps, N, dt, cands):
    ft = rb.make_file(amps, N, dt)
    p = Options().params(lib)
    buf = (nt.Candidate * max(cands.size, 1))()
    C.memmove(buf, cands.ctypes.data, cands.size * C.sizeof(nt.Candidate))
    cl = nt.CandidateList(C.cast(buf, C.POINTER(nt.Candidate)), cands.size, cands.size)
    res = lib.measure_ducy(C.byref(ft), C.byref(cl), C.byref(p))
    out = nt.candidates_to_numpy(res)["ducy"]
    lib.candlist_free(C.byref(res))
    return out


def test_ducy_golden_candidates(gpu_ready):
    path = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "small60.npz")))[0]
    z = np.load(path)
    amps, N, dt = z["amps"], int(z["N"]), float(z["dt"])
    cands = np.ascontiguousarray(z["raw"])
    ses = Session(N, dt, Options(blocksize=2048))
    ses.run_raw(amps)                       # the spectrum is now on the device
    got = ses.measure_ducy(cands)["ducy"]
    ses.close()
    host = _host_ducy(nt.host_lib(), amps, N, dt, cands)
    ref = _host_ducy(rb.ref_lib(), amps, N, dt, cands)
    np.testing.assert_array_equal(host, ref)
    np.testing.assert_array_equal(got, host)
    assert np.isfinite(got).all()


@pytest.mark.parametrize("nharms", [60, 32, 16])
def test_ducy_after_search(gpu_ready, nharms):
    """Collapsed candidates of a live search, edge cases included: a
    candidate whose harmonics run past Nyquist (short stack), one with no
    harmonic inside the spectrum (zero profile) and ones left NaN."""
    spec = synth.SeriesSpec(N=1 << 16, dt=64e-6, seed=21,
                            pulsars=[synth.Pulsar(23.7, 0.04, 30.0), synth.Pulsar(311.0, 0.08, 25.0)])
    amps = rb.ref_spectrum(synth.make_series(spec), spec.dt)
    opts = Options(nharms=nharms, blocksize=2048, threshold=6.0)
    ses = Session(spec.N, spec.dt, opts)
    cands = ses.collapse(ses.run_raw(amps))
    extra = np.zeros(4, dtype=nt.CAND_DTYPE)
    extra["r"] = [spec.N / 2 - 3.25, spec.N * 0.75, -2.0, 100.5]
    extra["nharm"] = [nharms, 4, 3, 0]
    extra["freq"] = extra["r"] / (spec.N * spec.dt)
    cands = np.concatenate([cands, extra])
    got = ses.measure_ducy(cands)["ducy"]
    ses.close()
    host = _host_ducy(nt.host_lib(), amps, spec.N, spec.dt, cands)
    np.testing.assert_array_equal(got, host)
    assert np.isnan(got[-2:]).all() and np.isfinite(got[:-2]).all()
