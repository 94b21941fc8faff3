"""Faults injected on the host into the spectrum reader (CPU): a missing or
incomplete .inf, a missing, empty or truncated .fft.  This build's
fftfile_open (libcoherent_search.so) and the reference's own
(src/fileio.c:52-139, compiled in oracle/_ref/libcsref.so) give the same
status and, when the file opens, the same N, bin count, T, DC and Nyquist."""
import ctypes as C
import os

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200 import synth

needs_ref = pytest.mark.skipif(not rb.have_ref(), reason="oracle/_ref not built")


def _open(lib, path):
    lib.fftfile_open.argtypes = [C.POINTER(nt.FFTFile), C.c_char_p]
    lib.fftfile_open.restype = C.c_int
    lib.fftfile_close.argtypes = [C.POINTER(nt.FFTFile)]
    ft = nt.FFTFile()
    rc = lib.fftfile_open(C.byref(ft), path.encode())
    fields = None
    if rc == 0:
        fields = (ft.N, ft.namps, ft.T, ft.DC, ft.Nyquist)
        lib.fftfile_close(C.byref(ft))
    return rc, fields


def _case(tmp, name, nbytes, inf):
    stem = os.path.join(tmp, name)
    if nbytes is not None:
        np.arange(nbytes, dtype=np.uint8).tofile(stem + ".fft")
    if inf == "full":
        synth.write_inf(stem + ".inf", 8192, 64e-6)
    elif inf == "no_n":
        with open(stem + ".inf", "w") as f:
            f.write(" Width of each time series bin (sec)    =  6.4e-05\n")
    elif inf == "no_dt":
        with open(stem + ".inf", "w") as f:
            f.write(" Number of bins in the time series      =  8192\n")
    return stem + ".fft"


CASES = {
    "complete": (8192 * 4, "full"),
    "missing_inf": (8192 * 4, None),
    "inf_without_N": (8192 * 4, "no_n"),
    "inf_without_dt": (8192 * 4, "no_dt"),
    "missing_fft": (None, "full"),
    "empty_fft": (0, "full"),
    "truncated_fft": (5000 * 8 + 5, "full"),       # fewer bins than N/2, odd byte count
    "longer_fft": (9000 * 8, "full"),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_fftfile_open_faults_match_reference(tmp_path, name):
    nbytes, inf = CASES[name]
    path = _case(str(tmp_path), name, nbytes, inf)
    ours = _open(nt.host_lib(), path)
    ref = _open(rb.ref_lib(), path)
    assert ours[0] == ref[0], (name, ours, ref)
    if name == "complete":
        assert ours[0] == 0
    if name in ("missing_inf", "inf_without_N", "inf_without_dt", "missing_fft"):
        assert ours[0] != 0
    if ours[0] == 0:
        assert ours[1][:3] == ref[1][:3]
        np.testing.assert_array_equal(np.array(ours[1][3:], np.float32),
                                      np.array(ref[1][3:], np.float32))
