"""The request loop (serve.SearchServer): requests of mixed lengths and
harmonic counts arrive as a Poisson stream while others run; each result is
identical to the same request searched alone, and to the plain
one-request-at-a-time server's."""
import numpy as np
import pytest

from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session
from coherentsearch_c_b200.serve import (PlainServer, Request, SearchServer, log_uniform_lengths,
                                         poisson_arrivals, run_stream)

pytestmark = pytest.mark.gpu
DT = 64e-6


def requests(n=12, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for i, N in enumerate(log_uniform_lengths(n, 1 << 14, 1 << 17, seed)):
        nh = int(rng.choice([16, 32, 60]))
        pulsars = [synth.Pulsar(float(rng.uniform(2, 40)), 0.05, 25.0)] if rng.random() < 0.5 else []
        x = synth.make_series(synth.SeriesSpec(N=N, dt=DT, seed=100 + i, pulsars=pulsars))
        amps = synth.amps_interleaved(synth.normalised_spectrum(x))
        out.append(Request(amps, N, DT, Options(nharms=nh, blocksize=4096, threshold=6.0)))
    return out


def alone(r):
    ses = Session(r.N, r.dt, r.opts)
    try:
        return ses.run_raw(r.amps)
    finally:
        ses.close()


def same(a, b):
    assert a.size == b.size
    for f in ("r", "metric", "nharm"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def test_stream_results_equal_alone(gpu_ready):
    reqs = requests()
    ref = [alone(r) for r in reqs]
    arrivals = poisson_arrivals(len(reqs), rate=2000.0, seed=1)   # many in flight at once
    with SearchServer(nslots=3) as srv:
        st = run_stream(srv, reqs, arrivals)
    for got, want in zip(st["results"], ref):
        same(got, want)
    assert st["p99_ms"] >= st["p50_ms"] > 0 and st["trials_per_s"] > 0
    with PlainServer() as plain:
        sp = run_stream(plain, reqs, arrivals)
    for got, want in zip(sp["results"], ref):
        same(got, want)
