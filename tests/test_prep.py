"""The raw-data front end on the GPU (prep.PrepSearch): dedispersed and
padded series bit-identical to the reference's prepsubband output, and each
DM's candidates equal to the reference's search of that series under the
search parity tolerances."""
import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200.prep import PrepSearch, running_mean
from coherentsearch_c_b200.search import Options

from test_dedisp import GEOMS, fb_for, ours_tables
from test_gpu_parity import SNR_RTOL_F32, match_candidates

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (rb.have_ref() and rb.have_dedisp_ref()),
                                 reason="oracle/_ref not built")]


def test_prep_search_matches_reference(gpu_ready):
    import torch
    g = GEOMS["c256_s16_d40"]
    dt = g[7]
    t = ours_tables(*g)
    raw = fb_for(g, nblocks=40, seed=11)
    numout = 24576
    opts = Options(blocksize=4096, threshold=6.0)
    ref_out = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                                t.blocks_per_read, numout)
    nout = ref_out.shape[1]
    pad = np.float32(running_mean(ref_out[0]))
    with PrepSearch(t, raw.shape[0], numout, dt, opts) as ps:
        d_raw = torch.from_numpy(raw).cuda()
        ps.dedisperse(d_raw.data_ptr(), raw.shape[0])
        assert ps.nout == nout and ps.pad_value == float(pad)
        single = {}
        for d in (0, 7, 13, 14, 25, 39):
            single[d] = ps.search_dm(d)
        # the pipelined loop over every DM (two sessions in turn)
        every = ps.search_all()
        assert len(every) == t.ndm
        for d in range(t.ndm):
            series = np.concatenate([ref_out[d], np.full(numout - nout, pad, np.float32)])
            np.testing.assert_array_equal(ps.series(d), series)
            amps = rb.ref_spectrum(series, dt)
            ref = rb.ref_search(amps, numout, dt, opts, collapse=False)
            got = every[d]
            if d in single:           # alone and in the pipelined loop: the same
                for f in ("freq", "metric", "r", "nharm"):
                    np.testing.assert_array_equal(single[d][f], got[f])
            match_candidates(got[np.argsort(got["freq"], kind="stable")], ref, opts.threshold,
                             SNR_RTOL_F32)
            if d == 25:   # search_file's post-processing on top
                refc = rb.ref_search(amps, numout, dt, opts, collapse=True)
                match_candidates(ps.ses.collapse(got), refc, opts.threshold, SNR_RTOL_F32)
        # the same loop collapsing on the GPU: the host collapse of the raw lists
        collapsed = ps.search_all(collapse=True)
        for d in range(t.ndm):
            host = ps.ses.collapse(every[d])
            assert collapsed[d].size == host.size
            for f in ("freq", "metric", "r", "nharm"):
                np.testing.assert_array_equal(collapsed[d][f], host[f])


def test_prep_search_clipped_matches_reference(gpu_ready):
    """The front end with prepsubband's default -clip 6 on a filterbank with
    RFI (bursts, a dropout spectrum, half the band saturated, a whole block of
    zeros): every DM's padded series bit for bit against the reference's
    clipped run, and its candidates -- raw, and collapsed on the GPU --
    against the reference's search of that series."""
    import torch
    from test_clip import _rfi
    g = GEOMS["c256_s16_d40"]
    dt = g[7]
    t = ours_tables(*g)
    raw = _rfi(fb_for(g, nblocks=40, seed=11), t.spectra_per_subint, flat_block=True)
    numout = 24576
    opts = Options(blocksize=4096, threshold=6.0)
    ref_out, nclip = rb.ref_dedisp_run(raw, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                                       t.blocks_per_read, numout, clip_sigma=6.0,
                                       return_clipped=True)
    assert nclip > t.spectra_per_subint                 # the zero block and the bursts
    nout = ref_out.shape[1]
    pad = np.float32(running_mean(ref_out[0]))
    with PrepSearch(t, raw.shape[0], numout, dt, opts) as ps:
        d_raw = torch.from_numpy(raw).cuda()
        ps.dedisperse(d_raw.data_ptr(), raw.shape[0])
        assert ps.nclipped == nclip and ps.nout == nout and ps.pad_value == float(pad)
        every = ps.search_all()
        collapsed = ps.search_all(collapse=True)
        for d in range(t.ndm):
            series = np.concatenate([ref_out[d], np.full(numout - nout, pad, np.float32)])
            np.testing.assert_array_equal(ps.series(d).view(np.uint32), series.view(np.uint32))
        for d in (0, 7, 20, 39):
            series = np.concatenate([ref_out[d], np.full(numout - nout, pad, np.float32)])
            amps = rb.ref_spectrum(series, dt)
            ref = rb.ref_search(amps, numout, dt, opts, collapse=False)
            got = every[d]
            match_candidates(got[np.argsort(got["freq"], kind="stable")], ref, opts.threshold,
                             SNR_RTOL_F32)
            refc = rb.ref_search(amps, numout, dt, opts, collapse=True)
            match_candidates(collapsed[d], refc, opts.threshold, SNR_RTOL_F32)
