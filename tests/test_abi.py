"""The drop-in boundary: the C-ABI libraries load and export exactly the
entry points declared in include/*.h (CPU; no compute call needs a GPU)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from coherentsearch_c_b200 import native as nt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared(header, prefix):
    text = open(os.path.join(INC, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(" + prefix + r"\w+)\s*\(", text))


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_gpu_library_exports_match_headers():
    lib = os.path.join(nt.LIBDIR, "libcsgpu.so")
    exp = exported(lib)
    want = declared("coherent_search.h", "cs_gpu_") | declared("cs_b200.h", "cs_b200_")
    want |= declared("cs_b200.h", "cs_gpu_")                  # the batch engine
    want |= declared("cs_b200.h", "cs_dedisp_") | declared("cs_b200.h", "cs_spectrum_")
    want |= declared("cs_b200.h", "cs_ducy_") | declared("cs_b200.h", "cs_clip_")
    assert want <= exp, sorted(want - exp)
    # nothing else leaks: the host helpers inside libcsgpu.so are hidden
    extra = {s for s in exp
             if not s.startswith(("cs_gpu_", "cs_b200_", "cs_dedisp_", "cs_spectrum_",
                                  "cs_ducy_", "cs_clip_"))}
    assert not extra, sorted(extra)


def test_host_library_exports_reference_api():
    exp = exported(os.path.join(nt.LIBDIR, "libcoherent_search.so"))
    want = {"params_defaults", "decimation_set", "direct_plans_build", "direct_plans_free",
            "trial_grid_rational", "chunk_starts", "cs_chunk_state", "cs_harmonic_fits",
            "harmonic_change_trials", "boxcar_widths", "ladder_boxcar_widths",
            "analytic_sigma", "boxcar_shape", "candlist_init", "candlist_free",
            "candlist_push", "remove_duplicates", "remove_harmonics", "write_candidates",
            "measure_ducy", "search_file", "search_cache_free", "fftfile_open",
            "fftfile_close", "inf_read", "cs_prep_pad_value", "cs_sigproc_read_header"}
    assert want <= exp, sorted(want - exp)


def test_libraries_load_and_report_no_gpu_here():
    gpu = nt.gpu_lib()
    nt.host_lib()
    buf = C.create_string_buffer(256)
    rc = gpu.cs_gpu_available(0, buf, 256)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert rc == -1 and buf.value
    else:
        assert rc == 1


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors (used to call both this build and the reference) have
    the layout the C compiler gives include/coherent_search.h."""
    checks = {"Candidate": ["freq", "metric", "r", "nharm", "ducy"],
              "CandidateList": ["v", "n", "cap"],
              "SearchParams": ["nharms", "hidr", "threshold", "ndecim", "decimations",
                               "precision", "sigma"],
              "DirectPlan": ["h", "dr0", "P", "row", "W", "carry", "ngrp", "gA_im"],
              "FFTFile": ["path", "inf", "N", "T", "DC", "amps", "namps", "owns_amps"]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "coherent_search.h"',
             'int main(void) {']
    for st, fields in checks.items():
        lines.append(f'printf("{st} size %zu\\n", sizeof({st}));')
        for f in fields:
            lines.append(f'printf("{st}.{f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "off.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "off"
    subprocess.run(["gcc", f"-I{INC}", str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True,
                                                         text=True, check=True).stdout.splitlines())
    for st, fields in checks.items():
        cls = getattr(nt, st)
        assert C.sizeof(cls) == int(out[f"{st} size"]), st
        for f in fields:
            assert getattr(cls, f).offset == int(out[f"{st}.{f}"]), (st, f)
