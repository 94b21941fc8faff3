"""SIGPROC filterbank files (cs_sigproc_read_header, coherentsearch_c_b200.sigproc):
the header PRESTO's reader parses (third_party/presto/src/sigproc_fb.c:240-345)
and the band edges it derives (:435-441), and the front end run from a file."""
import struct

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import sigproc, synth


def _spec(nchan=64, nspec=4800):
    return synth.FilterbankSpec(nchan=nchan, nspec=nspec, fctr=1400.0, bw=64.0, dt=128e-6,
                                dm=20.0, seed=5)


def test_header_round_trip(tmp_path):
    spec = _spec()
    raw = synth.make_filterbank(spec)
    path = tmp_path / "a.fil"
    synth.write_filterbank(str(path), raw, spec, source_name="J0000+00")
    h, data = sigproc.open_filterbank(str(path))
    assert h["nchans"] == spec.nchan and h["nbits"] == 8 and h["nifs"] == 1
    assert h["tsamp"] == spec.dt and h["source_name"] == "J0000+00"
    assert h["foff"] == -spec.chanwid and h["chanwid"] == spec.chanwid
    fch1 = spec.lofreq + (spec.nchan - 1) * spec.chanwid
    assert h["fch1"] == fch1
    assert h["lofreq"] == fch1 - (spec.nchan - 1) * spec.chanwid     # PRESTO's lo_freq
    assert h["nspectra"] == spec.nspec
    np.testing.assert_array_equal(np.asarray(data), raw)


def _write(path, keys):
    def s(x):
        b = x.encode()
        return struct.pack("<i", len(b)) + b
    with open(path, "wb") as f:
        f.write(s("HEADER_START"))
        for k, v in keys:
            f.write(s(k) + v)
        f.write(s("HEADER_END"))
        f.write(bytes(64 * 10))


@pytest.mark.parametrize("bad", ["nbits16", "foff_up", "unknown", "no_start"])
def test_header_refused(tmp_path, bad):
    keys = [("nchans", struct.pack("<i", 64)), ("nbits", struct.pack("<i", 8)),
            ("fch1", struct.pack("<d", 1500.0)), ("foff", struct.pack("<d", -1.0)),
            ("tsamp", struct.pack("<d", 64e-6))]
    if bad == "nbits16":
        keys[1] = ("nbits", struct.pack("<i", 16))
    elif bad == "foff_up":
        keys[3] = ("foff", struct.pack("<d", 1.0))
    elif bad == "unknown":
        keys.append(("not_a_keyword", struct.pack("<i", 1)))
    path = tmp_path / "b.fil"
    if bad == "no_start":
        with open(path, "wb") as f:
            f.write(b"\x00" * 64)
    else:
        _write(path, keys)
    with pytest.raises(ValueError):
        sigproc.read_header(str(path))


@pytest.mark.gpu
@pytest.mark.skipif(not rb.have_dedisp_ref(), reason="oracle/_ref not built")
def test_front_end_from_file(gpu_ready, tmp_path):
    """Tables from the file's header; dedispersed, padded series equal to the
    reference's block driver on the same file's samples."""
    import torch
    from coherentsearch_c_b200.prep import PrepSearch, running_mean
    from coherentsearch_c_b200.search import Options
    spec = _spec(nchan=128, nspec=16 * 2400)
    raw = synth.make_filterbank(spec)
    path = tmp_path / "c.fil"
    synth.write_filterbank(str(path), raw, spec)
    h, data = sigproc.open_filterbank(str(path))
    t = sigproc.dedisp_tables_for(h, nsub=16, ndm=12, lodm=0.0, dmstep=4.0)
    idisp, offs, bpr, _ = rb.ref_dedisp_tables(h["nchans"], 16, 12, 0.0, 4.0, h["lofreq"],
                                               h["chanwid"], h["tsamp"])
    np.testing.assert_array_equal(t.idispdt, idisp)
    np.testing.assert_array_equal(t.offsets, offs)
    numout = 1 << 15
    ref = rb.ref_dedisp_run(np.asarray(data), t.nsub, t.idispdt, t.offsets,
                            t.spectra_per_subint, t.blocks_per_read, numout)
    d = torch.from_numpy(np.array(data)).cuda()
    # this pulsar is nearly undispersed over 64 MHz, so prepsubband's default
    # 6-sigma clip cuts its pulses: the front end clips them as the reference does
    refc, nclip = rb.ref_dedisp_run(np.asarray(data), t.nsub, t.idispdt, t.offsets,
                                    t.spectra_per_subint, t.blocks_per_read, numout,
                                    clip_sigma=6.0, return_clipped=True)
    assert nclip > 0
    for clip, want_all in ((6.0, refc), (0.0, ref)):            # -clip 6, -noclip
        with PrepSearch(t, h["nspectra"], numout, h["tsamp"], Options(blocksize=4096),
                        clip_sigma=clip) as ps:
            ps.dedisperse(d.data_ptr(), h["nspectra"])
            assert ps.nclipped == (nclip if clip else 0)
            pad = np.float32(running_mean(want_all[0]))
            for dm in (0, 5, 11):
                want = np.concatenate([want_all[dm],
                                       np.full(numout - want_all.shape[1], pad, np.float32)])
                np.testing.assert_array_equal(ps.series(dm), want)
