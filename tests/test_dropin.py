"""Drop-in: the reference's own command-line programs, built as its GPU
configuration (-DCS_HAVE_CUDA) and linked against libcsgpu.so where the
reference links src/cuda.cu (oracle/Makefile target `dropin`).

The GPU tests run `coherent_search` and `coherent_search_list` from the
reference sources twice on the same seeded .dat inputs: once on the CPU
(stub build) and once with `--gpu 0` through this library.  That covers
realfft + rednoise, the search, collapse, the duty cycle and the .cohout
writer, all in the reference's own host code.  The .cohout files must list
the same candidates: frequencies, periods, harmonic counts and duty cycles
identical as printed, and S/N within the printed precision (0.01) plus
1e-4 relative.
"""
import os
import subprocess

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import synth

REF = os.path.join(rb.ROOT, "oracle", "_ref")
CPU_BIN = os.path.join(REF, "ref_coherent_search")
GPU_BIN = os.path.join(REF, "ref_coherent_search_b200")
CPU_LIST = os.path.join(REF, "ref_coherent_search_list")
GPU_LIST = os.path.join(REF, "ref_coherent_search_list_b200")

needs_dropin = pytest.mark.skipif(not (os.path.exists(GPU_BIN) and os.path.exists(CPU_BIN)),
                                  reason="oracle/_ref drop-in binaries not built")


def read_cohout(path):
    rows = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        f = line.split()
        rows.append((int(f[0]), float(f[1]), f[2], f[3], int(f[4]), f[5]))
    return rows


def same_cohout(a, b):
    ra, rb_ = read_cohout(a), read_cohout(b)
    assert len(ra) == len(rb_), (len(ra), len(rb_))
    assert len(ra) > 0
    for x, y in zip(ra, rb_):
        assert x[0] == y[0]
        assert x[2:] == y[2:], (x, y)          # freq, period, #harm, ducy as printed
        assert abs(x[1] - y[1]) <= 0.01 + 1e-4 * abs(y[1]), (x, y)


@needs_dropin
def test_dropin_links_this_library():
    out = subprocess.run(["ldd", GPU_BIN], capture_output=True, text=True, check=True).stdout
    line = [l for l in out.splitlines() if "libcsgpu.so" in l]
    assert line and os.path.join("coherentsearch_c_b200", "lib") in line[0], out


def _write(tmp, name, spec):
    x = synth.make_series(spec)
    return synth.write_dat(os.path.join(tmp, name), x, spec.dt)


def _run(cmd, cwd):
    p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, (cmd, p.returncode, p.stderr[-2000:])
    return p


@needs_dropin
@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small", "precision", "small_f64", "precision_f64"])
def test_reference_cli_on_gpu_matches_cpu(gpu_ready, tmp_path, case):
    """`*_f64` run both sides with --precision f64: the GPU side then takes
    the FP64 search (the reference's CPU f64 path is the FP64 oracle)."""
    if case.startswith("small"):
        spec = synth.config_small()
        extra = []
    else:
        spec = synth.config_precision(N=1 << 22)
        extra = ["--threads", str(min(16, os.cpu_count() or 1))]
    prec = ["--precision", "f64"] if case.endswith("_f64") else []
    dat = _write(str(tmp_path), case, spec)
    common = ["-t", "8", "--blocksize", "2048"] + prec
    _run([CPU_BIN] + common + extra + ["-o", "cpu.cohout", dat], str(tmp_path))
    _run([GPU_BIN, "--gpu", "0"] + common + ["-o", "gpu.cohout", dat], str(tmp_path))
    same_cohout(str(tmp_path / "gpu.cohout"), str(tmp_path / "cpu.cohout"))


@needs_dropin
@pytest.mark.gpu
def test_reference_list_cli_on_gpu_matches_cpu(gpu_ready, tmp_path):
    """List mode: uneven lengths, so the session is rebuilt per geometry and
    reused where the geometry repeats (cs_gpu_session_matches)."""
    names = []
    for i, (nlog, f0) in enumerate([(19, 11.2), (20, 11.2), (19, 5.3)]):
        spec = synth.SeriesSpec(N=1 << nlog, dt=64e-6, seed=500 + i,
                                pulsars=[synth.Pulsar(f0, 0.05, 25.0)])
        names.append(os.path.basename(_write(str(tmp_path), f"f{i}", spec)))
    (tmp_path / "sweep.dat.list").write_text("\n".join(names) + "\n")
    for exe, outdir, extra in ((CPU_LIST, "cpu", []), (GPU_LIST, "gpu", ["--gpu", "0"])):
        _run([exe] + extra + ["-t", "8", "--blocksize", "2048", "--outdir", outdir,
                              "sweep.dat.list"], str(tmp_path))
    for n in names:
        stem = os.path.splitext(n)[0]
        same_cohout(str(tmp_path / "gpu" / f"{stem}.cohout"),
                    str(tmp_path / "cpu" / f"{stem}.cohout"))
