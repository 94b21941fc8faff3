"""Time series -> normalised spectrum on the GPU (cs_spectrum_*): the
reference's in-memory realfft + rednoise (src/datpipe.c:101-253).

    with SpectrumMaker(N, dt) as sm:
        amps = sm.run(x)          # float32[N]: N/2 complex bins, FFTFile.amps layout
"""
from __future__ import annotations

import numpy as np

from . import native as nt


class SpectrumMaker:
    """A plan for series of N samples at sample time dt (one run at a time)."""

    def __init__(self, N: int, dt: float, startwidth: int = 6, endwidth: int = 100,
                 endfreq: float = 6.0, device: int = 0):
        self.N = int(N)
        self.lib = nt.gpu_lib()
        self.h = self.lib.cs_spectrum_create(self.N, dt, startwidth, endwidth, endfreq, device)
        if not self.h:
            raise RuntimeError("cs_spectrum_create failed (see stderr)")

    def run(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.size != self.N:
            raise ValueError(f"series of {x.size} samples for a plan of {self.N}")
        out = np.empty(self.N, dtype=np.float32)
        if self.lib.cs_spectrum_run(self.h, x.ctypes.data, out.ctypes.data) != 0:
            raise RuntimeError("cs_spectrum_run failed (see stderr)")
        return out

    def run_device(self, d_series: int, d_amps: int, stream: int | None = None) -> None:
        if self.lib.cs_spectrum_run_device(self.h, d_series, d_amps, stream) != 0:
            raise RuntimeError("cs_spectrum_run_device failed (see stderr)")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cs_spectrum_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
