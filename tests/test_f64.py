"""The FP64 search (--precision f64) on the GPU.

The reference's f64 mode interpolates in FP32 and widens the amplitudes, then
runs the c2r profile, the folds and the boxcar metric in double
(src/interp.c:555-573, src/search.c:288-292, 333-400, src/boxcar.c:715-731).
The GPU path keeps the FP32 interpolation bit for bit, so the only
difference left is the order of the FP64 sums of the profile transform
(the reference's FFT against a direct half-spectrum DFT here).

Tolerances (stated here, applied below):
  * every trial's metric: within 1e-9 of the oracle's FP64 metric, relative
    to the largest metric of the run;
  * candidates: r and harmonic count bit-exact, S/N within 1e-9 relative of
    the reference's own --precision f64 CPU path; a candidate on one side
    only must lie within 1e-9 (relative) of the threshold.
"""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session, search_spectrum

pytestmark = pytest.mark.gpu

F64_RTOL = 1e-9


def _case(seed=7, N=1 << 16, f0=37.3):
    spec = synth.SeriesSpec(N=N, dt=64e-6, seed=seed, pulsars=[synth.Pulsar(f0, 0.05, 30.0)])
    x = synth.make_series(spec)
    return spec, rb.ref_spectrum(x, spec.dt)


def match64(a, b, thr):
    ka = {(float(r), int(h)): float(m) for r, h, m in zip(a["r"], a["nharm"], a["metric"])}
    kb = {(float(r), int(h)): float(m) for r, h, m in zip(b["r"], b["nharm"], b["metric"])}
    for k in set(ka) & set(kb):
        assert abs(ka[k] - kb[k]) <= F64_RTOL * abs(kb[k]), (k, ka[k], kb[k])
    for k in set(ka) ^ set(kb):
        m = ka.get(k, kb.get(k))
        assert abs(m - thr) <= F64_RTOL * abs(thr), ("unmatched", k, m)


@pytest.mark.parametrize("nharms,hidr", [(60, 0.5), (32, 0.5), (16, 0.5), (7, 0.5),
                                         (16, 0.25)])
def test_f64_all_trial_metrics_vs_oracle(gpu_ready, nharms, hidr):
    """Every trial of every decimation slot against the oracle's FP64 metric,
    in the same (chunk, slot, trial) order."""
    spec, amps = _case()
    opts = Options(nharms=nharms, hidr=hidr, blocksize=2048, threshold=-1e30, remove=False,
                   harm_remove=False, precision=1)
    ses = Session(spec.N, spec.dt, opts)
    assert ses.info().kernel == 2
    raw = ses.run_raw(amps)
    ses.close()
    met, geo = rb.oracle_metrics(amps, spec.N, spec.dt, opts, 0, ses.total, prec64=True)
    ora = rb.oracle_candidates(met, geo, spec.N, spec.dt, opts)
    assert raw.size == ora.size
    np.testing.assert_array_equal(raw["r"], ora["r"])
    np.testing.assert_array_equal(raw["nharm"], ora["nharm"])
    d = np.abs(raw["metric"] - ora["metric"])
    assert d.max() <= F64_RTOL * max(1.0, np.abs(ora["metric"]).max()), d.max()


def test_f64_candidates_vs_reference_f64(gpu_ready):
    """Raw candidates of the FP64 GPU search against the reference CPU path
    run with --precision f64 (one OpenMP thread, its deterministic order)."""
    rb.pin_ref_threads(1)
    spec, amps = _case()
    opts = Options(blocksize=2048, threshold=6.0, precision=1)
    ref = rb.ref_search(amps, spec.N, spec.dt, opts, precision=1, collapse=False)
    ses = Session(spec.N, spec.dt, opts)
    raw = ses.run_raw(amps)
    ses.close()
    assert ref.size > 50
    raw = raw[np.argsort(raw["freq"], kind="stable")]
    match64(raw, ref, 6.0)


def test_f64_config_small_end_to_end(gpu_ready):
    """search_file with precision f64 on the N = 2^20 configuration: the
    collapsed list equals the reference's f64 run."""
    rb.pin_ref_threads(1)
    x = synth.make_series(synth.config_small())
    amps = rb.ref_spectrum(x, 64e-6)
    opts = Options(blocksize=2048, threshold=8.0, precision=1)
    ref64 = rb.ref_search(amps, x.size, 64e-6, opts, precision=1)
    got = search_spectrum(amps, x.size, 64e-6, opts)
    match64(got, ref64, 8.0)
    assert np.any(np.abs(got["freq"] - 7.3) < 0.01)
