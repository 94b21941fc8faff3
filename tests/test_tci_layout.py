"""The tensor-core interpolation's decomposition, restated on the CPU.

tci::interp_tc (cs_interp_tc.cuh) computes every (trial, harmonic) value as
a product over bands: for trial t = c q + i (pnum 1) and harmonic h, with the
band of NB positions i0 <= i < i0 + NB that holds i,

    X_h(t) = sum_kk Bh[i - i0][kk] . amp[base_h + c h + R_h(i0) + kk]

where Bh folds the row's gain into its weights (tci_load in cs_gpu.cu).  This
test restates that construction from the reference planner's DirectPlan
tables and checks, in float64, that it equals the reference's per-trial
formula (src/cuda.cu:97-135: window from the residue table, sum of m taps,
then the rotation by the gain) for every trial of the first and last column
tiles of the three default configurations, and that every band window fits
the kernel's K (<= 64 halves).
"""
import ctypes as C

import numpy as np
import pytest

import refbind as rb
from coherentsearch_c_b200 import native as nt
from coherentsearch_c_b200.search import Options

NB, KMAX, M = 24, 64, 16


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
        out.append(dict(
            rfloor0=dp.rfloor0, q=q, P=P, pnum=dp.pnum,
            row=np.ctypeslib.as_array(dp.row, shape=(q,)).copy(),
            carry=np.ctypeslib.as_array(dp.carry, shape=(P,)).copy(),
            W=np.ctypeslib.as_array(dp.W, shape=(P * M,)).reshape(P, M).astype(np.float64),
            Are=np.ctypeslib.as_array(dp.A_re, shape=(P,)).astype(np.float64),
            Aim=np.ctypeslib.as_array(dp.A_im, shape=(P,)).astype(np.float64)))
    lib.direct_plans_free(C.byref(plans))
    return out, total


def _direct(pl, h, t, amp):
    """The reference's per-trial value (float64)."""
    q = pl["q"]
    qint, res = divmod(t * h * pl["pnum"], q)
    ph = pl["row"][res] - 1
    b0 = pl["rfloor0"] + qint + int(pl["carry"][ph]) + 1 - M // 2
    win = amp[b0:b0 + M]
    s = (pl["W"][ph] * win).sum()
    gr, gi = pl["Are"][ph], pl["Aim"][ph]
    return complex(gr * s.real - gi * s.imag, gr * s.imag + gi * s.real)


@pytest.mark.parametrize("nh,N", [(60, 1 << 20)])
def test_band_products_equal_reference_formula(nh, N):
    opts = Options(nharms=nh)
    plans, total = _plans(N, 64e-6, opts)
    rng = np.random.default_rng(5)
    namps = N // 2
    amp = rng.standard_normal(namps) + 1j * rng.standard_normal(namps)
    for h, pl in enumerate(plans, start=1):
        q, P = pl["q"], pl["P"]
        assert pl["pnum"] == 1 and q % NB == 0
        reach = np.nonzero(pl["row"] > 0)[0]
        cres = pl["carry"][pl["row"][reach] - 1]
        carry_res = int(reach[np.argmax(cres)]) if cres.any() else q

        def R(i):
            return (i * h) // q + (((i * h) % q) >= carry_res)

        base = pl["rfloor0"] + 1 - M // 2
        ncol = total // q
        for c in (0, 1, ncol // 2, ncol - 1):
            for b in range(q // NB):
                i0 = b * NB
                rel = R(i0)
                wb = R(i0 + NB - 1) - rel + M
                assert (2 * wb + 15) // 16 * 16 <= KMAX
                w0 = base + c * h + rel
                if w0 < 0 or w0 + wb > namps:
                    continue
                window = amp[w0:w0 + wb]
                for i in range(i0, i0 + NB):
                    ph = i % P
                    gr, gi = pl["Are"][ph], pl["Aim"][ph]
                    kk = R(i) - rel + np.arange(M)
                    # the band row with the gain folded in (Re, Im outputs)
                    re = (gr * pl["W"][ph] * window[kk].real - gi * pl["W"][ph] * window[kk].imag).sum()
                    im = (gi * pl["W"][ph] * window[kk].real + gr * pl["W"][ph] * window[kk].imag).sum()
                    want = _direct(pl, h, c * q + i, amp)
                    assert abs(complex(re, im) - want) <= 1e-9 * max(1.0, abs(want)), (h, c, i)
