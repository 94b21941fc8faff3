"""The host library under AddressSanitizer and UndefinedBehaviorSanitizer
(CPU only).  tests/host_sanitize.c drives planning, tables, the record sort
and harvest, the boxcar tables, candidate post-processing, the .cohout writer
and reader, measure_ducy and the .fft/.inf and SIGPROC readers; any
sanitizer report fails the test."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from coherentsearch_c_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "coherentsearch_c_b200", "csrc")
HOST_SRCS = [os.path.join(CSRC, "host", f) for f in ("cs_common.c", "cs_search.c", "cs_tables.c")]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_host_library_under_sanitizers(tmp_path):
    exe = str(tmp_path / "host_sanitize")
    subprocess.run(["gcc", "-std=gnu11", "-g", "-O1", "-fno-omit-frame-pointer",
                    "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
                    "-ffp-contract=off", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}",
                    os.path.join(ROOT, "tests", "host_sanitize.c"), *HOST_SRCS, "-o", exe,
                    "-lm"], check=True, capture_output=True)
    # inputs: a .fft/.inf pair and a small SIGPROC filterbank
    rng = np.random.default_rng(5)
    stem = str(tmp_path / "spec")
    rng.standard_normal(2 * 4096).astype(np.float32).tofile(stem + ".fft")
    synth.write_inf(stem + ".inf", 8192, 64e-6)
    spec = synth.FilterbankSpec(nchan=64, nspec=2000, fctr=1400.0, bw=64.0, seed=3)
    fil = str(tmp_path / "small.fil")
    synth.write_filterbank(fil, synth.make_filterbank(spec), spec)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    out = subprocess.run([exe, str(tmp_path), stem + ".fft", fil], capture_output=True,
                         text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-4000:]
    assert "runtime error" not in out.stderr, out.stderr[-4000:]
    assert "host_sanitize: ok" in out.stdout
