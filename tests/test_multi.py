"""Several spectra in one persistent launch (cs_b200_multi_enqueue).

The multi-spectrum kernel runs the warp-specialised search body over one
list of (spectrum, tile) work items; each tile takes its own spectrum's
tables, operand scale and record buffer.  Every spectrum's candidates must
equal those of its own single-spectrum search, bit for bit (same kernel
body, same arithmetic), in lists of uneven lengths where CTAs straddle
spectra.
"""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import MultiGraph, Options, Session, multi_search

pytestmark = pytest.mark.gpu


def _spectra(lengths, seed0=900):
    out = []
    for i, nlog in enumerate(lengths):
        spec = synth.SeriesSpec(N=1 << nlog, dt=64e-6, seed=seed0 + i,
                                pulsars=[synth.Pulsar(11.2 + i, 0.05, 25.0)])
        out.append((spec.N, rb.ref_spectrum(synth.make_series(spec), spec.dt)))
    return out


@pytest.mark.parametrize("nh", [60, 32, 16])
def test_multi_launch_equals_single_searches(gpu_ready, monkeypatch, nh):
    monkeypatch.delenv("CS_B200_GENERIC_KERNEL", raising=False)
    monkeypatch.delenv("CS_B200_TMA_KERNEL", raising=False)
    data = _spectra([16, 18, 17, 16, 19])
    opts = Options(nharms=nh, blocksize=2048, threshold=6.0)
    single = []
    sessions = []
    for N, amps in data:
        ses = Session(N, 64e-6, opts)
        assert ses.info().kernel == 1
        single.append(ses.run_raw(amps))        # also leaves the spectrum on the device
        sessions.append(ses)
    try:
        for _ in range(2):                      # twice: reused tables, cleared counters
            got, _ = multi_search(sessions)
            assert len(got) == len(single)
            for a, b in zip(got, single):
                assert a.size == b.size and a.size > 0
                np.testing.assert_array_equal(a["r"], b["r"])
                np.testing.assert_array_equal(a["nharm"], b["nharm"])
                np.testing.assert_array_equal(a["metric"], b["metric"])
    finally:
        for s in sessions:
            s.close()


def test_multi_launch_refuses_mixed_configurations(gpu_ready):
    data = _spectra([16, 16])
    s60 = Session(data[0][0], 64e-6, Options(nharms=60, blocksize=2048))
    s32 = Session(data[1][0], 64e-6, Options(nharms=32, blocksize=2048))
    try:
        with pytest.raises(RuntimeError):
            multi_search([s60, s32])
    finally:
        s60.close()
        s32.close()


def test_multi_graph_replays_equal_multi_launch(gpu_ready, monkeypatch):
    """The launch recorded as a CUDA graph gives, replay after replay, the
    candidates of cs_b200_multi_enqueue on the same spectra; a session whose
    record buffer grew makes the graph refuse to replay."""
    monkeypatch.delenv("CS_B200_GENERIC_KERNEL", raising=False)
    monkeypatch.delenv("CS_B200_TMA_KERNEL", raising=False)
    data = _spectra([16, 18, 17, 16, 19], seed0=940)
    opts = Options(nharms=60, blocksize=2048, threshold=6.0)
    sessions = []
    for N, amps in data:
        ses = Session(N, 64e-6, opts)
        assert ses.info().kernel == 1
        ses.run_raw(amps)
        sessions.append(ses)
    try:
        ref, _ = multi_search(sessions)
        g = MultiGraph(sessions)
        try:
            for _ in range(3):
                got, _ = g.search()
                for a, b in zip(got, ref):
                    assert a.size == b.size and a.size > 0
                    np.testing.assert_array_equal(a["r"], b["r"])
                    np.testing.assert_array_equal(a["nharm"], b["nharm"])
                    np.testing.assert_array_equal(a["metric"], b["metric"])
        finally:
            g.close()
        # every valid (trial, slot) is recorded at this threshold: the 2^19
        # spectrum's record buffer overflows and grows
        g = MultiGraph(sessions, threshold=-1e30)
        try:
            g.launch()
            rcs = [s.collect(-1e30)[2] for s in sessions]
            assert rcs[4] == 1
            with pytest.raises(MultiGraph.StaleGraph):
                g.launch()
        finally:
            g.close()
    finally:
        for s in sessions:
            s.close()
