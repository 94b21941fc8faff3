"""Batched search (cs_gpu_batch_*): every request's result equals the same
spectrum searched alone through cs_gpu_session_run -- same candidates, same
order, same S/N bits -- whatever else runs beside it, however the slots'
device buffers are reused, and under a device-memory budget."""
import numpy as np
import pytest

from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.batch import Batch
from coherentsearch_c_b200.search import Options, Session

pytestmark = pytest.mark.gpu

DT = 64e-6
# (log2 N, nharms, seed): lengths and harmonic counts mixed, so slots switch
# geometry and kernel (nharms 60 takes the warp-specialised kernel)
MIX = [(17, 60, 1), (15, 32, 2), (16, 60, 3), (17, 16, 4), (15, 60, 5), (16, 32, 6),
       (17, 60, 1)]


def spectrum(nlog, seed):
    spec = synth.SeriesSpec(N=1 << nlog, dt=DT, seed=seed,
                            pulsars=[synth.Pulsar(9.7 + seed, 0.05, 25.0)])
    return synth.amps_interleaved(synth.normalised_spectrum(synth.make_series(spec)))


def opts_for(nh):
    return Options(nharms=nh, blocksize=4096, threshold=6.0)


def alone(amps, nlog, nh):
    ses = Session(1 << nlog, DT, opts_for(nh))
    try:
        return ses.run_raw(amps)
    finally:
        ses.close()


def same(a, b):
    assert a.size == b.size
    for f in ("r", "freq", "metric", "nharm"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.fixture(scope="module")
def cases():
    out = []
    for nlog, nh, seed in MIX:
        amps = spectrum(nlog, seed)
        out.append((nlog, nh, amps, alone(amps, nlog, nh)))
    assert all(c[3].size > 0 for c in out)
    return out


@pytest.mark.parametrize("nslots", [1, 3])
def test_batch_matches_single_runs(gpu_ready, cases, nslots):
    with Batch(nslots=nslots) as b:
        ids = [b.submit(amps, 1 << nlog, DT, opts_for(nh)) for nlog, nh, amps, _ in cases]
        assert b.pending() == len(ids)
        for rid, (_, _, _, ref) in zip(ids, cases):
            got, queued, run = b.wait(rid)
            same(got, ref)
            assert queued >= 0 and run > 0
        assert b.pending() == 0


def test_batch_under_memory_budget(gpu_ready, cases):
    """A budget that holds about one request at a time: slots give buffers
    back and wait, and the results do not change."""
    big = max(c[2].nbytes for c in cases)
    budget = big * 3 + (24 << 20)
    with Batch(nslots=3, mem_budget=budget) as b:
        assert b.device_bytes() == 0
        ids = [b.submit(amps, 1 << nlog, DT, opts_for(nh)) for nlog, nh, amps, _ in cases]
        for rid, (_, _, _, ref) in zip(ids, cases):
            same(b.wait(rid)[0], ref)
            assert b.device_bytes() > 0         # sessions kept for reuse


def test_batch_rejects_request_beyond_budget(gpu_ready, cases):
    nlog, nh, amps, _ = cases[0]
    with Batch(nslots=2, mem_budget=1 << 20) as b:
        rid = b.submit(amps, 1 << nlog, DT, opts_for(nh))
        with pytest.raises(RuntimeError):
            b.wait(rid)


def test_batch_warm_then_serve(gpu_ready, cases):
    """Slots loaded ahead for the largest request (nharms 60, a longer
    spectrum than any case) serve every case with unchanged results; the
    load-only requests leave nothing pending."""
    with Batch(nslots=3) as b:
        b.warm(1 << 18, DT, opts_for(60))
        assert b.pending() == 0
        ids = [b.submit(amps, 1 << nlog, DT, opts_for(nh)) for nlog, nh, amps, _ in cases]
        for rid, (_, _, _, ref) in zip(ids, cases):
            same(b.wait(rid)[0], ref)
        b.warm(1 << 15, DT, opts_for(16))           # smaller: reuses the buffers
        rid = b.submit(cases[0][2], 1 << cases[0][0], DT, opts_for(cases[0][1]))
        same(b.wait(rid)[0], cases[0][3])


def test_batch_cancel(gpu_ready, cases):
    """One slot, many requests: the queued ones can be cancelled (their wait
    raises BatchCancelled), a finished one cannot, and the others' results do
    not change."""
    from coherentsearch_c_b200.batch import BatchCancelled
    with Batch(nslots=1) as b:
        ids = [b.submit(amps, 1 << nlog, DT, opts_for(nh)) for nlog, nh, amps, _ in cases]
        cancelled = [b.cancel(rid) for rid in ids[3:]]
        assert any(cancelled)                   # the last ones were still queued
        for rid, (_, _, _, ref), c in zip(ids, cases, [False] * 3 + cancelled):
            if c:
                with pytest.raises(BatchCancelled):
                    b.wait(rid)
            else:
                same(b.wait(rid)[0], ref)
        assert b.pending() == 0
        rid = b.submit(cases[0][2], 1 << cases[0][0], DT, opts_for(cases[0][1]))
        same(b.wait(rid)[0], cases[0][3])
        with pytest.raises(KeyError):
            b.cancel(rid)                        # already waited for
