"""bench.py's CPU legs, run here without a GPU at a small size.

The reference arm (`--impl reference`) and the CPU baseline forms time the
reference's own CPU path compiled from its sources (oracle/_ref/libcsref.so).
These tests check the arm's JSON contract and that the single-thread and
process-per-core forms run and report; the numbers themselves are only
meaningful on the GPU box's host.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcsref.so"))

pytestmark = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref/libcsref.so not built")


def test_reference_arm_json_contract():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "3", "--nlog2", "17"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
              "cpu_baseline"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] >= 3
    assert "N=2^17" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_cpu_reference_forms_run_and_report():
    sys.path.insert(0, ROOT)
    import bench
    from coherentsearch_c_b200 import synth
    N = 1 << 17
    x = synth.make_series(synth.config_precision(N=N))
    amps = synth.amps_interleaved(synth.normalised_spectrum(x))
    forms = bench.cpu_reference_forms(amps, N, nproc=2)
    assert forms["one_thread"]["cores"] == 1 and forms["one_thread"]["value"] > 0
    # the timed build of the reference: its FFT shim's share of the search
    assert forms["one_thread"]["fft_calls"] > 0
    assert 0.0 < forms["one_thread"]["fft_share"] < 1.0
    assert forms["processes"]["cores"] == 2 and forms["processes"]["value"] > 0
    assert "2 single-threaded processes" in forms["processes"]["sample"]
