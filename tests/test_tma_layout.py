"""Index arithmetic of the column-tile kernel (cs_search_tma.cuh), on the CPU.

The kernel finds every trial's interpolation window from column-tile
offsets instead of the reference's per-trial residue walk.  This test
restates its arithmetic in numpy and checks, for every trial of the three
default configurations, that

  * the window start equals the reference's (src/cuda.cu:97-116 through the
    reference planner's own DirectPlan tables);
  * the window lies inside the staged TMA box row (22 bins) and inside the
    nine 16-byte reads the lane makes from it;
  * every trial belongs to exactly one (round, TMEM quarter, buffer, lane);
  * the box coordinates are even, non-negative, and every element a box row
    reads lies inside the padded spectrum copy.
"""
import ctypes as C

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200.search import Options

M = 16
BOXW, ROWS, FRONT, BACK = 22, 16, 64, 2048


def _plans(N, dt, opts):
    lib = rb.ref_lib()
    p = opts.params(lib)
    r_lo, lodr, total = opts.geometry(N, dt)
    plans = nt.DirectPlanSet()
    assert lib.direct_plans_build(C.byref(plans), C.byref(p), r_lo) == 0
    out = []
    for h in range(1, opts.nharms + 1):
        dp = plans.plans[h - 1]
        q, P = dp.q, dp.P
        row = np.ctypeslib.as_array(dp.row, shape=(q,)).copy()
        carry = np.ctypeslib.as_array(dp.carry, shape=(P,)).copy()
        out.append((dp.rfloor0, dp.pnum, q, row, carry))
    lib.direct_plans_free(C.byref(plans))
    return out, total


@pytest.mark.parametrize("nh,N", [(60, 1 << 23), (32, 1 << 21), (16, 1 << 20)])
def test_column_tile_windows_match_reference(nh, N):
    opts = Options(nharms=nh)
    plans, total = _plans(N, 64e-6, opts)
    namps = N // 2
    # (t*h)//q = (t//q)*h + ((t%q)*h)//q exactly, so the per-trial identities
    # repeat every column tile: check the first and last 64 column tiles
    span = 64 * 2 * nh
    t = np.unique(np.concatenate([np.arange(min(span, total)),
                                  np.arange(max(0, total - span), total)])).astype(np.int64)
    for h, (rfloor0, pnum, q, row, carry) in enumerate(plans, start=1):
        assert pnum == 1 and q == 2 * nh and q % 8 == 0
        # the reference's window start for every trial
        tp = t * h
        qint, res = tp // q, tp % q
        b0_ref = rfloor0 + qint + carry[row[res] - 1] + 1 - M // 2
        # carry as a residue threshold, monotone over the residues harmonic h
        # reaches (row[r] == 0 marks the others)
        reach = np.nonzero(row > 0)[0]
        cres = carry[row[reach] - 1]
        assert np.all(np.diff(cres.astype(int)) >= 0)
        carry_res = int(reach[np.argmax(cres)]) if cres.any() else q

        def R(i):
            return (i * h) // q + ((i * h) % q >= carry_res)

        c, i = t // q, t % q
        x_kernel = rfloor0 - M // 2 + 1 + c * h + R(i)
        np.testing.assert_array_equal(x_kernel, b0_ref)
        # the round (8 trials of 32 column tiles), quarter, buffer and lane
        sup, i0 = c // 32, (i // 8) * 8
        quarter, buf = (i - i0) // 2, (i - i0) % 2
        nsup = ((total - 1) // q + 32) // 32
        assert quarter.max() == 3 and buf.max() == 1 and sup.max() < nsup
        rowstart = rfloor0 - M // 2 + 1 + c * h + R(i0)
        off = b0_ref - rowstart
        assert off.min() >= 0 and (off + M).max() <= BOXW
        # the lane's nine float4 reads start at the even bin at or below the
        # first trial of its pair and cover both windows
        oa = R(i0 + 2 * quarter) - R(i0)
        first = 2 * (oa >> 1)
        assert np.all(oa <= 3)
        assert np.all(off >= first) and np.all(off + M <= first + 18)
        assert np.all(first + 18 <= BOXW)
        # box coordinates of both parity classes of every round
        sv, uv = np.meshgrid(np.arange(nsup), np.arange(q // 8), indexing="ij")
        xa = rfloor0 - M // 2 + 1 + 32 * sv * h + R(8 * uv) + FRONT
        dim0_bins = namps + FRONT + BACK - 30 * h
        for cls in (0, 1):
            xs = xa + cls * h
            x0 = xs - (xs & 1)
            assert x0.min() >= 0 and np.all(x0 % 2 == 0)
            # the last element of the last row lies inside the padded copy,
            # unless it is past the map's inner extent (zero-filled, not read)
            last = x0 + BOXW - 1
            inside = last < dim0_bins
            assert np.all(last[inside] + 2 * h * (ROWS - 1) < namps + FRONT + BACK)
