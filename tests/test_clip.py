"""prepsubband's time-domain clipping on the device -- the replaced spectra
(cs_clip_count, cs_clip_levels), the channel levels written over them and the
clipped dedispersion (cs_dedisp_run_device_clipped) -- against the reference's
own clip_times run in its block driver, bit for bit, and the front end that
runs it."""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200.dedisp import Dedisperser, dedisp_tables

from test_dedisp import GEOMS, fb_for, ours_tables

needs_ref = pytest.mark.skipif(not rb.have_dedisp_ref(), reason="oracle/_ref not built")


def _ref(raw, t, clip):
    return rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                             t.blocks_per_read, clip_sigma=clip, return_clipped=True)


def _rfi(raw, L, flat_block=False):
    nb = raw.shape[0] // L
    raw = raw.copy()
    b1, b2, b3 = nb // 6, nb // 2, (5 * nb) // 6
    raw[b1 * L + 100: b1 * L + 104, :] = 255         # a broadband burst of four spectra
    raw[b2 * L + 7, :] = 0                           # a dropout
    raw[b3 * L + 300, ::2] = 255                     # half the band saturated
    if flat_block:
        # a whole block of zeros (a receiver dropout): no sample lies strictly
        # inside median -+ 3 sigma = 0, so the block has no good spectra and
        # keeps the running statistics and channel levels (clipping.c:139-144)
        raw[(nb // 3) * L:(nb // 3 + 1) * L, :] = 0
    return raw


@needs_ref
def test_reference_clipping_leaves_clean_data_alone():
    """The pin the device path relies on: with nothing clipped, the clipped
    run is the unclipped run, bit for bit (CPU)."""
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=40, seed=11)
    plain = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                              t.blocks_per_read)
    clipped, n = _ref(raw, t, 6.0)
    assert n == 0
    np.testing.assert_array_equal(plain, clipped)
    rfi, n = _ref(_rfi(raw, t.spectra_per_subint), t, 6.0)
    assert n > 0


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("geom,nblocks", [("c256_s16_d40", 40), ("c200_s8_d25_cps25", 30),
                                          ("filterbank_1024x64x500", 8)])
def test_clip_count_matches_reference(gpu_ready, geom, nblocks):
    import torch
    g = GEOMS[geom]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=nblocks, seed=3)
    L = t.spectra_per_subint
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        for data in (raw, _rfi(raw, L)):
            _, want = _ref(data, t, 6.0)
            d = torch.from_numpy(np.ascontiguousarray(data)).cuda()
            got = dd.clip_count(d.data_ptr(), data.shape[0], 6.0)
            torch.cuda.synchronize()
            assert got == want, (geom, got, want)
            # with caller-kept scratch, twice (nothing carries over between calls)
            scr = torch.empty(dd.clip_scratch_bytes(data.shape[0]), dtype=torch.uint8,
                              device="cuda")
            for _ in range(2):
                assert dd.clip_count(d.data_ptr(), data.shape[0], 6.0, None, scr.data_ptr(),
                                     scr.numel()) == want
        # a lower threshold clips more, in both
        data = _rfi(raw, L)
        _, want = _ref(data, t, 3.0)
        d = torch.from_numpy(np.ascontiguousarray(data)).cuda()
        assert dd.clip_count(d.data_ptr(), data.shape[0], 3.0) == want


def _device_clipped(dd, t, raw, clip=6.0, numout=-1):
    """Flags, levels and the clipped dedispersion of raw on the GPU."""
    import torch
    L = t.spectra_per_subint
    nspec = raw.shape[0]
    nblk = nspec // L
    d = torch.from_numpy(np.ascontiguousarray(raw)).cuda()
    flags = torch.full((nblk * L,), 7, dtype=torch.uint8, device="cuda")
    levels = torch.full((nblk, t.nchan), float("nan"), dtype=torch.float32, device="cuda")
    n = dd.clip_levels(d.data_ptr(), nspec, flags.data_ptr(), levels.data_ptr(), clip)
    nout = dd.output_length(nspec, numout)
    stride = (nout + 3) // 4 * 4
    out = torch.full((t.ndm, stride), -1.0, dtype=torch.float32, device="cuda")
    got = dd.run_device_clipped(d.data_ptr(), nspec, flags.data_ptr(), levels.data_ptr(),
                                out.data_ptr(), stride, numout)
    torch.cuda.synchronize()
    assert got == nout
    return n, flags.cpu().numpy(), levels.cpu().numpy(), out.cpu().numpy()[:, :nout]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("geom,nblocks,numout", [("c256_s16_d40", 40, -1),
                                                 ("c200_s8_d25_cps25", 30, -1),
                                                 ("c64_s64_d7", 30, -1),
                                                 ("filterbank_1024x64x500", 8, -1),
                                                 ("c256_s16_d40", 40, 9000)])
@pytest.mark.parametrize("kernel", ["ws", "rounds"])
def test_clipped_dedispersion_matches_reference(gpu_ready, monkeypatch, geom, nblocks, numout,
                                                kernel):
    """prepsubband -clip on the GPU: the replaced spectra, the channel levels
    written over them (clip_times' good_chan_levels after every block) and the
    dedispersed series, all bit for bit against the reference's own run --
    through the warp-specialised DM stage and through the rounds kernel it
    falls back to (CS_B200_DEDISP_ROUNDS)."""
    if kernel == "rounds":
        monkeypatch.setenv("CS_B200_DEDISP_ROUNDS", "1")
    else:
        monkeypatch.delenv("CS_B200_DEDISP_ROUNDS", raising=False)
    g = GEOMS[geom]
    t = ours_tables(*g)
    raw = _rfi(fb_for(g, nblocks=nblocks, seed=3), t.spectra_per_subint,
               flat_block=geom != "filterbank_1024x64x500")
    want, nref, lev = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                                        t.blocks_per_read, numout, clip_sigma=6.0,
                                        return_clipped=True, return_levels=True)
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        n, flags, levels, out = _device_clipped(dd, t, raw, numout=numout)
    read = ~np.isnan(lev).any(axis=1)                  # blocks the reference read
    if numout < 0:
        assert read.all()
        assert n == nref > 0
    assert set(np.unique(flags)) <= {0, 1} and int(flags.sum()) == n
    np.testing.assert_array_equal(levels[:, ::-1][read].view(np.uint32),
                                  lev[read].view(np.uint32))
    assert out.shape == want.shape
    np.testing.assert_array_equal(out.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_clipped_path_without_clips_is_the_integer_path(gpu_ready, geom):
    """Nothing flagged: the float sums in the reference's order give the
    integer path's bits (every partial sum is an integer below 2^24)."""
    import torch
    g = GEOMS[geom]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=12, seed=5)
    L = t.spectra_per_subint
    nspec = raw.shape[0]
    with Dedisperser(t, max_spectra=nspec) as dd:
        plain = dd.run(raw)
        nout = plain.shape[1]
        stride = (nout + 3) // 4 * 4
        d = torch.from_numpy(raw).cuda()
        flags = torch.zeros(nspec // L * L, dtype=torch.uint8, device="cuda")
        levels = torch.full((nspec // L, t.nchan), 1e30, dtype=torch.float32, device="cuda")
        out = torch.empty((t.ndm, stride), dtype=torch.float32, device="cuda")
        assert dd.run_device_clipped(d.data_ptr(), nspec, flags.data_ptr(), levels.data_ptr(),
                                     out.data_ptr(), stride) == nout
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy()[:, :nout].view(np.uint32),
                                      plain.view(np.uint32))


@pytest.mark.gpu
@needs_ref
def test_front_end_clips_like_the_reference(gpu_ready):
    """PrepSearch with prepsubband's default -clip 6: the padded series of
    every DM equal the reference's clipped run; with clip_sigma=0 (-noclip)
    the unclipped one."""
    import torch
    from coherentsearch_c_b200.prep import PrepSearch, running_mean
    from coherentsearch_c_b200.search import Options
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = _rfi(fb_for(g, nblocks=40, seed=11), t.spectra_per_subint)
    numout = 24576
    d = torch.from_numpy(raw).cuda()
    for clip in (6.0, 0.0):
        want, nref = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                                       t.blocks_per_read, numout, clip_sigma=clip,
                                       return_clipped=True)
        with PrepSearch(t, raw.shape[0], numout, g[7], Options(blocksize=4096),
                        clip_sigma=clip) as ps:
            ps.dedisperse(d.data_ptr(), raw.shape[0])
            torch.cuda.synchronize()
            assert ps.nclipped == nref and (nref > 0) == (clip > 0)
            got = ps.out.cpu().numpy()
            nout = want.shape[1]
            assert ps.nout == nout
            np.testing.assert_array_equal(got[:, :nout].view(np.uint32), want.view(np.uint32))
            pad = np.float32(running_mean(want[0]))
            assert (got[:, nout:ps.N] == pad).all()


@pytest.mark.gpu
def test_clip_levels_edge_cases(gpu_ready):
    """Less than one block: nothing is decided or written; clip_sigma 0 (-noclip)
    writes nothing either; a clipped run with no complete output chunk writes no
    output."""
    import torch
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    L = t.spectra_per_subint
    raw = fb_for(g, nblocks=3, seed=2)
    with Dedisperser(t, max_spectra=raw.shape[0]) as dd:
        d = torch.from_numpy(np.ascontiguousarray(raw)).cuda()
        flags = torch.full((3 * L,), 7, dtype=torch.uint8, device="cuda")
        levels = torch.full((3, t.nchan), -1.0, dtype=torch.float32, device="cuda")
        for nspec, clip in ((L - 1, 6.0), (0, 6.0), (raw.shape[0], 0.0)):
            assert dd.clip_levels(d.data_ptr(), nspec, flags.data_ptr(), levels.data_ptr(),
                                  clip) == 0
        torch.cuda.synchronize()
        assert (flags.cpu().numpy() == 7).all() and (levels.cpu().numpy() == -1.0).all()
        # one block: decisions and levels for it, but no output chunk completes
        assert dd.output_length(L) == 0
        n = dd.clip_levels(d.data_ptr(), L, flags.data_ptr(), levels.data_ptr(), 6.0)
        out = torch.full((t.ndm, 4), -1.0, dtype=torch.float32, device="cuda")
        assert dd.run_device_clipped(d.data_ptr(), L, flags.data_ptr(), levels.data_ptr(),
                                     out.data_ptr(), 4) == 0
        torch.cuda.synchronize()
        assert n == 0 and (out.cpu().numpy() == -1.0).all()
        assert set(np.unique(flags.cpu().numpy()[:L])) == {0}
        assert (flags.cpu().numpy()[L:] == 7).all()
