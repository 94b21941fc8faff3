"""Session reuse through the reference ABI: cs_gpu_session_free parks the
session and the next cs_gpu_session_create reloads it for a new geometry.
A reloaded session returns the same candidates, bit for bit, as one made
fresh -- across lengths, harmonic counts and the two kernels."""
import numpy as np
import pytest

from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.search import Options, Session

pytestmark = pytest.mark.gpu

DT = 64e-6
# (log2 N, nharms): lengths and harmonic counts change from file to file
FILES = [(18, 60), (16, 32), (17, 60), (15, 16), (18, 60), (16, 7)]


def spectrum(nlog, seed):
    spec = synth.SeriesSpec(N=1 << nlog, dt=DT, seed=seed,
                            pulsars=[synth.Pulsar(7.3 + seed, 0.05, 25.0)])
    return synth.amps_interleaved(synth.normalised_spectrum(synth.make_series(spec)))


def search(amps, nlog, nh):
    ses = Session(1 << nlog, DT, Options(nharms=nh, blocksize=8192, threshold=6.0))
    try:
        return ses.run_raw(amps)
    finally:
        ses.close()


def test_reloaded_sessions_match_fresh_ones(gpu_ready):
    gpu = nt.gpu_lib()
    spectra = [spectrum(nlog, i) for i, (nlog, _) in enumerate(FILES)]
    fresh = []
    for (nlog, nh), amps in zip(FILES, spectra):
        gpu.cs_b200_session_park_drain()           # a new session every time
        fresh.append(search(amps, nlog, nh))
    gpu.cs_b200_session_park_drain()
    for _ in range(2):                             # each create reloads a parked one
        for (nlog, nh), amps, want in zip(FILES, spectra, fresh):
            got = search(amps, nlog, nh)
            assert got.size == want.size > 0
            for f in ("r", "freq", "metric", "nharm"):
                np.testing.assert_array_equal(got[f], want[f], err_msg=f)
    assert 1 <= gpu.cs_b200_session_park_drain() <= 2
    assert gpu.cs_b200_session_park_drain() == 0


def test_park_off_frees_at_once(gpu_ready):
    """CS_B200_SESSION_PARK=0: cs_gpu_session_free releases the session, as
    the reference's does (the limit is read once per process, so a child
    process runs it)."""
    import os
    import subprocess
    import sys
    code = (
        "import numpy as np\n"
        "from coherentsearch_c_b200 import native as nt\n"
        "from coherentsearch_c_b200.search import Options, Session\n"
        "amps = np.ones(1 << 15, np.float32)\n"
        "for _ in range(3):\n"
        "    s = Session(1 << 15, 64e-6, Options(nharms=16, blocksize=8192))\n"
        "    s.run_raw(amps)\n"
        "    s.close()\n"
        "print(nt.gpu_lib().cs_b200_session_park_drain())\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for park, want in (("0", "0"), ("1", "1")):
        env = dict(os.environ, CS_B200_SESSION_PARK=park, PYTHONPATH=root)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                             text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        assert out.stdout.strip().splitlines()[-1] == want, (park, out.stdout)
