"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference CPU search path compiled from the reference sources
(oracle/_ref/libcsref.so, built by `make -C oracle ref`) on seeded synthetic
inputs and stores inputs and outputs as small .npz files.  The fixtures pin
the oracle and the GPU path without needing the reference at test time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import refbind as rb  # noqa: E402
from coherentsearch_c_b200 import synth  # noqa: E402
from coherentsearch_c_b200.search import Options  # noqa: E402

CASES = {
    # name: (series spec, options)
    "small60": (synth.SeriesSpec(N=1 << 15, dt=64e-6, seed=101,
                                 pulsars=[synth.Pulsar(41.3, 0.04, 28.0)]),
                dict(nharms=60, blocksize=2048, threshold=6.0)),
    "small32": (synth.SeriesSpec(N=1 << 15, dt=64e-6, seed=102,
                                 pulsars=[synth.Pulsar(17.9, 0.06, 25.0)]),
                dict(nharms=32, blocksize=1024, threshold=6.0)),
    "small16_hidr025": (synth.SeriesSpec(N=1 << 14, dt=128e-6, seed=103,
                                         pulsars=[synth.Pulsar(9.1, 0.08, 22.0)]),
                        dict(nharms=16, hidr=0.25, blocksize=512, threshold=5.5, maxdecim=4)),
}


def fields(opts):
    return {k: np.array(v) for k, v in opts.items()}


def main():
    if not rb.have_ref():
        raise SystemExit("build the reference first: make -C oracle ref")
    for name, (spec, o) in CASES.items():
        opts = Options(**o)
        x = synth.make_series(spec)
        amps = rb.ref_spectrum(x, spec.dt)
        raw = rb.ref_search(amps, spec.N, spec.dt, opts, collapse=False)
        col = rb.ref_search(amps, spec.N, spec.dt, opts, collapse=True)
        raw64 = rb.ref_search(amps, spec.N, spec.dt, opts, precision=1, collapse=False)
        r_lo, lodr, total, cstarts = rb.ref_chunks(amps, spec.N, spec.dt, opts)
        extra = {"series": x} if name == "small16_hidr025" else {}
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), amps=amps, N=spec.N, dt=spec.dt, **extra,
            raw=raw, collapsed=col, raw64=raw64, cstarts=cstarts, total=total,
            r_lo=r_lo, lodr=lodr, **{"opt_" + k: v for k, v in fields(o).items()})
        print(name, "raw", raw.size, "collapsed", col.size, "total", total)


if __name__ == "__main__":
    main()
