"""Parity at the benchmarked configuration.

bench.py times one search of the precision-study spectrum: N = 2^23 float32
samples at dt = 64 us (three pulsars at 1.7, 29.4 and 311 Hz on red noise),
nharms 60, m 16, hidr 0.5, 0.1-125 Hz, decimations 1..6, blocksize 65536,
threshold 8 -- 8,046,622 trials through the warp-specialised tensor-core
kernel, with its 65,536-trial chunks and 32-bit trial positions.  This test
searches exactly that spectrum through cs_gpu_session_run, FP32 and FP64,
and compares both with the reference's own CPU path (compiled from its
sources, one OpenMP thread so its chunk order is deterministic) run at the
same blocksize in f32 and in --precision f64.

Tolerances (the GPU parity tests' own):
  * r and harmonic count bit-exact;
  * FP32 GPU S/N within 1e-4 relative of the reference f32 path and within
    1e-3 of its f64 path (the FP64 oracle);
  * FP64 GPU S/N within 1e-9 relative of the reference f64 path;
  * a candidate on one side only must lie within the band of its tolerance
    around the threshold.

CS_B200_PRECISION_TABLE=<path> also writes the per-candidate table (the
collapsed candidates with their S/N in each arithmetic) as JSON.
"""
import json
import os

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session

pytestmark = pytest.mark.gpu

THR = 8.0
N_BENCH = 1 << 23
DT = 64e-6


def _match(a, b, rtol, band):
    ka = {(float(r), int(h)): float(m) for r, h, m in zip(a["r"], a["nharm"], a["metric"])}
    kb = {(float(r), int(h)): float(m) for r, h, m in zip(b["r"], b["nharm"], b["metric"])}
    worst = 0.0
    for k in set(ka) & set(kb):
        rel = abs(ka[k] - kb[k]) / abs(kb[k])
        worst = max(worst, rel)
        assert rel <= rtol, (k, ka[k], kb[k])
    flips = set(ka) ^ set(kb)
    for k in flips:
        m = ka.get(k, kb.get(k))
        assert abs(m - THR) <= band * THR, ("unmatched", k, m)
    return worst, len(flips)


@pytest.fixture(scope="module")
def bench_case():
    x = synth.make_series(synth.config_precision(N=N_BENCH))
    amps = synth.amps_interleaved(synth.normalised_spectrum(x))
    assert x.size == N_BENCH
    return amps


def _by_freq(c):
    return c[np.argsort(c["freq"], kind="stable")]


def test_bench_config_matches_reference(gpu_ready, bench_case):
    amps = bench_case
    opts = Options(nharms=60, m=16, blocksize=65536, threshold=THR)
    opts64 = Options(nharms=60, m=16, blocksize=65536, threshold=THR, precision=1)

    ses = Session(N_BENCH, DT, opts)
    assert ses.total == 8046622
    assert ses.info().kernel in (1, 3)              # the benchmarked kernel family
    raw = ses.run_raw(amps)                         # (chunk, slot, j) order
    col = ses.collapse(raw)
    raw = _by_freq(raw)
    ses.close()
    ses64 = Session(N_BENCH, DT, opts64)
    assert ses64.info().kernel == 2
    raw64 = ses64.run_raw(amps)
    col64 = ses64.collapse(raw64)
    raw64 = _by_freq(raw64)
    ses64.close()

    rb.pin_ref_threads(1)
    ref = rb.ref_search(amps, N_BENCH, DT, opts, collapse=False)
    ref64 = rb.ref_search(amps, N_BENCH, DT, opts, precision=1, collapse=False)
    refc64 = rb.ref_search(amps, N_BENCH, DT, opts, precision=1)
    assert ref.size > 1000                          # strong sources, many raw candidates

    w32, f32 = _match(raw, ref, 1e-4, 1e-3)
    w32_64, f32_64 = _match(raw, ref64, 1e-3, 1e-3)
    w64, f64 = _match(raw64, ref64, 1e-9, 1e-9)
    _match(col64, refc64, 1e-9, 1e-9)
    _match(col, refc64, 1e-3, 1e-3)
    # every injected pulsar inside the band is found (311 Hz only as k >= 3)
    for f0 in (1.7, 29.4, 311.0):
        assert np.any(np.abs(col["freq"] - f0) < 0.01 * f0), f0

    path = os.environ.get("CS_B200_PRECISION_TABLE")
    if path:
        k64 = {(float(r), int(h)): float(m) for r, h, m in
               zip(col64["r"], col64["nharm"], col64["metric"])}
        kref = {(float(r), int(h)): float(m) for r, h, m in
                zip(refc64["r"], refc64["nharm"], refc64["metric"])}
        rows = []
        for c in col:
            k = (float(c["r"]), int(c["nharm"]))
            rows.append({"freq_hz": float(c["freq"]), "nharm": int(c["nharm"]),
                         "snr_f32_gpu": float(c["metric"]), "snr_f64_gpu": k64.get(k),
                         "snr_f64_ref_cpu": kref.get(k)})
        with open(path, "w") as f:
            json.dump({"raw_candidates": int(raw.size),
                       "max_rel_snr_err_f32_vs_ref_f32": w32,
                       "max_rel_snr_err_f32_vs_ref_f64": w32_64,
                       "max_rel_snr_err_f64_vs_ref_f64": w64,
                       "flips_f32_vs_ref_f32": f32, "flips_f32_vs_ref_f64": f32_64,
                       "flips_f64_vs_ref_f64": f64, "collapsed": rows}, f, indent=1)
