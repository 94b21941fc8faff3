"""Candidate harvest and collapse on the GPU (cs_b200_session_collect_collapsed)
against the same post-processing on the host (src/search.c:1467-1478:
remove_duplicates or a stable frequency sort, then remove_harmonics) of the
same raw candidates: identical lists, for every combination of the two
switches, small and large candidate counts."""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session
from test_gpu_parity import SNR_RTOL_F32, match_candidates

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")]


def _spectrum(seed=21, N=1 << 16):
    spec = synth.SeriesSpec(N=N, dt=64e-6, seed=seed,
                            pulsars=[synth.Pulsar(23.7, 0.04, 30.0), synth.Pulsar(311.0, 0.08, 25.0)])
    return spec, rb.ref_spectrum(synth.make_series(spec), spec.dt)


def _same(a, b):
    assert a.size == b.size, (a.size, b.size)
    for f in ("freq", "metric", "r", "nharm"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def _device_vs_host(ses, amps):
    ses.run_raw(amps)                     # uploads the spectrum
    ses.enqueue(None)
    raw, _, rc = ses.collect()
    assert rc == 0
    ses.enqueue(None)
    dev, _, rc = ses.collect_collapsed()
    assert rc == 0
    host = ses.collapse(raw)
    _same(dev, host)
    return raw, dev


@pytest.mark.parametrize("nharms", [60, 32, 16])
@pytest.mark.parametrize("remove,harm_remove", [(True, True), (True, False), (False, True),
                                                (False, False)])
def test_collapse_matches_host(gpu_ready, nharms, remove, harm_remove):
    spec, amps = _spectrum()
    opts = Options(nharms=nharms, blocksize=2048, threshold=5.0, remove=remove,
                   harm_remove=harm_remove)
    ses = Session(spec.N, spec.dt, opts)
    raw, dev = _device_vs_host(ses, amps)
    ses.close()
    assert raw.size > 200
    if remove or harm_remove:
        assert dev.size < raw.size


def test_collapse_matches_reference(gpu_ready):
    """search_file's own post-processing on the reference's candidates: the
    same collapsed list within the S/N tolerance."""
    spec, amps = _spectrum(seed=5)
    opts = Options(blocksize=2048, threshold=6.0)
    ses = Session(spec.N, spec.dt, opts)
    ses.run_raw(amps)
    ses.enqueue(None)
    dev, _, rc = ses.collect_collapsed()
    ses.close()
    ref = rb.ref_search(amps, spec.N, spec.dt, opts, collapse=True)
    match_candidates(dev, ref, 6.0, SNR_RTOL_F32)
    assert abs(dev.size - ref.size) <= 1


def test_collapse_many_candidates(gpu_ready):
    """Tens of thousands of raw candidates (a low threshold on a strong
    source): long duplicate runs and a long greedy pass."""
    spec, amps = _spectrum(seed=9, N=1 << 18)
    opts = Options(blocksize=8192, threshold=2.5)
    ses = Session(spec.N, spec.dt, opts)
    raw, dev = _device_vs_host(ses, amps)
    ses.close()
    assert raw.size > 20000 and 0 < dev.size < raw.size


def test_collapse_empty(gpu_ready):
    spec, amps = _spectrum()
    ses = Session(spec.N, spec.dt, Options(blocksize=2048, threshold=1e9))
    ses.run_raw(amps)
    ses.enqueue(None, 1e9)
    dev, _, rc = ses.collect_collapsed(1e9)
    ses.close()
    assert rc == 0 and dev.size == 0
