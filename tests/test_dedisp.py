"""Subband dedispersion (cs_dedisp_*) against the reference.

The reference here is PRESTO's dispersion.c as vendored by the reference
(delay tables, dedisp_subbands, float_dedisp), compiled with its -Ofast
flags, driven block by block as src/prep_dedisp.c's get_data loop drives it
(oracle/dedisp_harness.c).  Requirements: delay tables identical; every
output sample of every DM bit-identical (float32 bits) to the reference's;
output length identical.

CPU tests pin the tables and the harness itself (against the absolute-time
formula); GPU tests run the kernels.
"""
import ctypes as C

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200 import synth
from coherentsearch_c_b200.dedisp import Dedisperser, dedisp_tables, output_length

needs_ref = pytest.mark.skipif(not rb.have_dedisp_ref(), reason="oracle/_ref not built")

FB = synth.config_filterbank(nspec=1 << 16)

# (nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, L)
GEOMS = {
    "filterbank_1024x64x500": (1024, 64, 500, 0.0, 0.4, FB.lofreq, FB.chanwid, 64e-6, 2400),
    "c256_s16_d40": (256, 16, 40, 10.0, 1.5, 1200.0, 1.0, 128e-6, 600),
    "c200_s8_d25_cps25": (200, 8, 25, 0.0, 3.0, 400.0, 0.5, 256e-6, 1200),
    "c64_s64_d7": (64, 64, 7, 0.0, 20.0, 800.0, 0.5, 64e-6, 800),
}
# 150 MHz and DMs to 250: offsets of ~70,000 samples, wider than shared memory
WIDE = (64, 64, 7, 100.0, 25.0, 150.0, 0.125, 64e-6, 800)


def ours_tables(nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, L):
    return dedisp_tables(nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, L)


def formula(raw, nsub, idisp, offs, nout):
    """S_s[T] = sum_c X_c[T + d_c]; out_d[T] = sum_s S_s[T + off_ds] (int64)."""
    x = raw[:, ::-1].astype(np.int64).T                       # [nchan][nspec], ascending
    nchan, nspec = x.shape
    cps = nchan // nsub
    ns = nout + int(offs.max()) + 1
    S = np.zeros((nsub, ns), np.int64)
    for c in range(nchan):
        d = int(idisp[c])
        S[c // cps] += x[c, d:d + ns]
    out = np.zeros((offs.shape[0], nout), np.int64)
    for dm in range(offs.shape[0]):
        for s in range(nsub):
            o = int(offs[dm, s])
            out[dm] += S[s, o:o + nout]
    return out


def fb_for(geom, nblocks, seed=1):
    nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, L = geom
    spec = synth.FilterbankSpec(nchan=nchan, nspec=nblocks * L + L // 3,
                                fctr=lofreq - 0.5 * chanwid + 0.5 * chanwid * nchan,
                                bw=chanwid * nchan, dt=dt, dm=lodm + dmstep * ndm / 3,
                                f0=7.7, seed=seed)
    return synth.make_filterbank(spec)


@needs_ref
@pytest.mark.parametrize("name", list(GEOMS) + ["wide"])
def test_tables_match_reference(name):
    g = GEOMS.get(name, WIDE)
    t = ours_tables(*g)
    idisp, offs, bpr, avg = rb.ref_dedisp_tables(*g[:8], L=g[8])
    np.testing.assert_array_equal(t.idispdt, idisp)
    np.testing.assert_array_equal(t.offsets, offs)
    assert t.blocks_per_read == bpr
    assert t.avgdm == avg


@needs_ref
def test_reference_harness_matches_formula():
    """The restated block driver around the reference's kernels gives the
    absolute-time formula exactly, with the reference's output length."""
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=9)
    ref = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                            t.blocks_per_read)
    n = output_length(t, raw.shape[0])
    assert ref.shape == (t.ndm, n) and n > 0
    f = formula(raw, t.nsub, t.idispdt, t.offsets, n)
    np.testing.assert_array_equal(ref, f.astype(np.float32))


@needs_ref
@pytest.mark.parametrize("nblocks,numout", [(4, -1), (5, -1), (9, -1), (9, 1000), (9, 0),
                                            (2, -1), (13, 3601)])
def test_output_length_matches_reference(nblocks, numout):
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=nblocks, seed=nblocks)
    ref = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                            t.blocks_per_read, numout)
    assert ref.shape[1] == output_length(t, raw.shape[0], numout)


def test_library_exports_dedisp_and_rejects_bad_tables():
    lib = nt.gpu_lib()
    bad = (C.c_int * 4)()
    assert lib.cs_dedisp_tables(10, 3, 1, 0.0, 1.0, 1400.0, 1.0, 1e-4, 2400, bad, bad, None,
                                None) == -1      # 10 channels do not split into 3 subbands


# ---------------------------------------------------------------- GPU ---
@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name,nblocks,numout", [
    ("c256_s16_d40", 11, -1), ("c256_s16_d40", 11, 2000), ("c200_s8_d25_cps25", 10, -1),
    ("c64_s64_d7", 14, -1), ("filterbank_1024x64x500", 12, -1)])
def test_gpu_bit_exact(gpu_ready, name, nblocks, numout):
    g = GEOMS[name]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=nblocks, seed=7)
    ref = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                            t.blocks_per_read, numout)
    assert ref.shape[1] > 0
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        for _ in range(2):                      # the plan is reusable
            got = dd.run(raw, numout)
            assert got.shape == ref.shape
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


@needs_ref
@pytest.mark.gpu
def test_gpu_device_entry_point_matches_host(gpu_ready):
    import torch
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=11, seed=9)
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        host = dd.run(raw)
        n = host.shape[1]
        d_raw = torch.from_numpy(raw).cuda()
        stride = (n + 3) // 4 * 4 + 4
        d_out = torch.full((t.ndm, stride), -1.0, device="cuda")
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            got = dd.run_device(d_raw.data_ptr(), raw.shape[0], d_out.data_ptr(), stride,
                                stream=stream.cuda_stream)
        stream.synchronize()
        assert got == n
        out = d_out.cpu().numpy()
        np.testing.assert_array_equal(out[:, :n], host)
        assert (out[:, n:] == -1.0).all()       # nothing written past the output
        sb, dm = dd.last_times()
        assert sb > 0 and dm > 0


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("direct", [False, True])
def test_gpu_offsets_wider_than_shared_memory(gpu_ready, monkeypatch, direct):
    """Offsets of ~70,000 samples: the staged kernel runs groups of one DM;
    the direct kernel (the plan's choice when not even one DM's windows fit
    in shared memory, forced here by CS_B200_DEDISP_DIRECT) gives the same
    bits."""
    if direct:
        monkeypatch.setenv("CS_B200_DEDISP_DIRECT", "1")
    else:
        monkeypatch.delenv("CS_B200_DEDISP_DIRECT", raising=False)
    t = ours_tables(*WIDE)
    nb = 3 * t.blocks_per_read + 2
    raw = fb_for(WIDE, nblocks=nb, seed=3)
    ref = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                            t.blocks_per_read)
    assert ref.shape[1] > 0
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        got = dd.run(raw)
    np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_gpu_rejects_delays_beyond_block(gpu_ready):
    lib = nt.gpu_lib()
    idisp = np.full(16, 3000, np.int32)         # more than one 2400-spectrum block
    offs = np.zeros((1, 4), np.int32)
    ip = C.POINTER(C.c_int)
    plan = lib.cs_dedisp_create(16, 4, 1, idisp.ctypes.data_as(ip), offs.ctypes.data_as(ip),
                                2400, 1, 10000, 0)
    assert not plan
