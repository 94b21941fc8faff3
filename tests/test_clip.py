"""prepsubband's time-domain clipping: the device count of replaced spectra
(cs_clip_count) against the reference's own clip_times run in the block
driver, and the front end's refusal when clipping would act."""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200.dedisp import Dedisperser, dedisp_tables

from test_dedisp import GEOMS, fb_for, ours_tables

needs_ref = pytest.mark.skipif(not rb.have_dedisp_ref(), reason="oracle/_ref not built")


def _ref(raw, t, clip):
    return rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                             t.blocks_per_read, clip_sigma=clip, return_clipped=True)


def _rfi(raw, L):
    nb = raw.shape[0] // L
    raw = raw.copy()
    b1, b2, b3 = nb // 6, nb // 2, (5 * nb) // 6
    raw[b1 * L + 100: b1 * L + 104, :] = 255         # a broadband burst of four spectra
    raw[b2 * L + 7, :] = 0                           # a dropout
    raw[b3 * L + 300, ::2] = 255                     # half the band saturated
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


@pytest.mark.gpu
@needs_ref
def test_front_end_refuses_when_clipping_would_act(gpu_ready):
    import torch
    from coherentsearch_c_b200.prep import PrepSearch
    from coherentsearch_c_b200.search import Options
    g = GEOMS["c256_s16_d40"]
    t = ours_tables(*g)
    raw = _rfi(fb_for(g, nblocks=40, seed=11), t.spectra_per_subint)
    with PrepSearch(t, raw.shape[0], 24576, g[7], Options(blocksize=4096)) as ps:
        d = torch.from_numpy(raw).cuda()
        with pytest.raises(RuntimeError, match="clip"):
            ps.dedisperse(d.data_ptr(), raw.shape[0])
    with PrepSearch(t, raw.shape[0], 24576, g[7], Options(blocksize=4096), clip_sigma=0) as ps:
        ps.dedisperse(d.data_ptr(), raw.shape[0])      # -noclip: runs
