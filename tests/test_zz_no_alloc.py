"""cs_b200_session_search_noalloc against cs_gpu_session_run (GPU).

The entry point runs the session's kernels with per-call scratch in a static
device array instead of session buffers.  Two consecutive calls must each
give the candidates of the allocating path: same positions, harmonic counts
and order, S/N within 1e-6 relative (the kernels are the same; the records
only travel a different route).  Collected last so that it also runs after
every other GPU test in one process.
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200.search import Options, Session

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-6
MAX_RECS = 65536          # CS_B200_NOALLOC_MAX_RECS in include/cs_b200.h
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _case(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    o = {k[4:]: z[k].item() for k in z.files if k.startswith("opt_")}
    return z["amps"], int(z["N"]), float(z["dt"]), Options(**o)


def noalloc(ses, thr, cap, d_amps=None):
    out = np.zeros(max(cap, 1), dtype=nt.CAND_DTYPE)
    n = C.c_longlong(-1)
    rc = ses.gpu.cs_b200_session_search_noalloc(ses.sess, d_amps, thr, out.ctypes.data, cap,
                                                C.byref(n), None)
    return rc, out[:max(n.value, 0)]


def same(got, want):
    assert got.size == want.size
    np.testing.assert_array_equal(got["r"], want["r"])
    np.testing.assert_array_equal(got["freq"], want["freq"])
    np.testing.assert_array_equal(got["nharm"], want["nharm"])
    np.testing.assert_allclose(got["metric"], want["metric"], rtol=SNR_RTOL)


@pytest.mark.parametrize("name,generic", [("small60", False), ("small60", True),
                                          ("small32", True)])
def test_noalloc_matches_session_run(gpu_ready, monkeypatch, name, generic):
    if generic:
        monkeypatch.setenv("CS_B200_GENERIC_KERNEL", "1")
    else:
        monkeypatch.delenv("CS_B200_GENERIC_KERNEL", raising=False)
    amps, N, dt, opts = _case(name)
    ses = Session(N, dt, opts)
    try:
        want = ses.run_raw(amps)        # allocating path; leaves amps on the device
        assert want.size > 0
        for _ in range(2):
            rc, got = noalloc(ses, opts.threshold, want.size + 64)
            assert rc == 0
            same(got, want)
        # an explicit device pointer and a second, higher threshold
        rc, got = noalloc(ses, opts.threshold + 1.0, want.size + 64, ses.device_amps_ptr())
        assert rc == 0
        same(got, want[want["metric"] > opts.threshold + 1.0])
    finally:
        ses.close()


def test_noalloc_rejects_beyond_limits(gpu_ready, monkeypatch):
    monkeypatch.delenv("CS_B200_GENERIC_KERNEL", raising=False)
    amps, N, dt, opts = _case("small60")
    ses = Session(N, dt, opts)
    try:
        want = ses.run_raw(amps)
        assert ses.total * ses.info().nslot > MAX_RECS
        rc, got = noalloc(ses, -1e30, MAX_RECS + 1)      # every record passes
        assert rc == -2 and got.size == 0
        rc, got = noalloc(ses, opts.threshold, 0)         # no room for the records
        assert rc == -3 and got.size == 0
        rc, got = noalloc(ses, opts.threshold, want.size + 64)   # and nothing left behind
        assert rc == 0
        same(got, want)
    finally:
        ses.close()
