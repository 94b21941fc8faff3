"""The raw-data front end on one GPU: 8-bit filterbank -> subband
dedispersion -> for every DM, the series padded to `numout` points ->
realfft + rednoise -> coherent search, as the reference's
prep_coherent_search runs it (src/prep_dedisp.c:484-522, 744-790;
src/prep_search.c) without clipping, masking, downsampling or barycentring.

Every stage stays on the device: the dedispersed series are written into a
[ndm][numout] buffer, padded there, turned into spectra in a session's device
buffer and searched; only candidates come back.  All DMs share one geometry,
so one search session (tables built once) serves them all.
"""
from __future__ import annotations

import numpy as np

from .dedisp import Dedisperser, DedispTables
from .search import Options, Session
from .spectrum import SpectrumMaker


def running_mean(x: np.ndarray) -> float:
    """The one-pass mean of PRESTO's update_stats over x (float32), in
    double -- the padding value prepsubband writes (cs_prep_pad_value)."""
    import ctypes as C
    from . import native as nt
    x = np.ascontiguousarray(x, dtype=np.float32)
    return float(nt.host_lib().cs_prep_pad_value(x.ctypes.data_as(C.POINTER(C.c_float)), x.size))


class PrepSearch:
    """Dedisperse a filterbank and search every DM series on one GPU.

    Two search sessions of the one geometry alternate over the DMs: while DM
    d is searched on one, DM d+1's spectrum is made on the prep stream into
    the other's spectrum buffer and DM d-1's candidates are read back."""

    def __init__(self, tables: DedispTables, nspec: int, numout: int, dt: float,
                 opts: Options | None = None, device: int = 0):
        import torch
        self.torch = torch
        self.t = tables
        self.dt = dt
        self.opts = opts or Options()
        self.dev = f"cuda:{device}"
        self.dd = Dedisperser(tables, max_spectra=nspec, device=device)
        self.nout = self.dd.output_length(nspec, numout)
        if self.nout <= 0:
            raise ValueError("no complete output chunk for this many spectra")
        # the searched length: numout points (data + padding), even
        self.N = int(numout) - (int(numout) & 1)
        self.stride = (self.N + 3) // 4 * 4
        self.out = torch.empty((tables.ndm, self.stride), dtype=torch.float32, device=self.dev)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.spec = SpectrumMaker(self.N, dt, device=device)
        self.sessions = [Session(self.N, dt, self.opts, device=device) for _ in range(2)]
        self.ses = self.sessions[0]
        self.pad_value = None
        self.search_ms: list[float] = []     # search kernel time of each DM, last pass

    def dedisperse(self, d_raw: int, nspec: int) -> None:
        """Dedisperse [nspec][nchan] uint8 at device address d_raw, then pad
        every series from nout to N with DM 0's running mean."""
        torch = self.torch
        # the raw block may still be in flight on the caller's stream
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))
        n = self.dd.run_device(d_raw, nspec, self.out.data_ptr(), self.stride, self.N,
                               self.stream.cuda_stream)
        if n != self.nout:
            raise RuntimeError(f"dedispersion wrote {n} samples per DM, expected {self.nout}")
        if self.nout < self.N:
            with torch.cuda.stream(self.stream):
                head = self.out[0, :self.nout].to("cpu", non_blocking=False)
            self.pad_value = float(np.float32(running_mean(head.numpy())))
            with torch.cuda.stream(self.stream):
                self.out[:, self.nout:self.N].fill_(self.pad_value)

    def _spectrum(self, d: int, ses: Session) -> None:
        self.spec.run_device(self.out[d].data_ptr(), ses.device_amps_ptr(),
                             self.stream.cuda_stream)

    def _finish(self, ses: Session, threshold: float | None, collapse: bool = False) -> np.ndarray:
        get = ses.collect_collapsed if collapse else ses.collect
        out, ms, rc = get(threshold)
        if rc == 1:                     # record buffer grown: run again
            ses.enqueue(None, threshold)
            out, ms, rc = get(threshold)
        self.search_ms.append(ms)
        return out

    def search_dm(self, d: int, threshold: float | None = None) -> np.ndarray:
        """Spectrum and search of DM d's series: raw candidates."""
        ses = self.sessions[0]
        self._spectrum(d, ses)
        ses.enqueue(None, threshold, after_stream=self.stream.cuda_stream)
        return self._finish(ses, threshold)

    def search_all(self, threshold: float | None = None, dms=None,
                   collapse: bool = False) -> list[np.ndarray]:
        """Candidates of every DM (or of `dms`), pipelined over the two
        sessions, in DM order: raw, or with `collapse` the list search_file
        returns, collapsed on the GPU."""
        dms = list(range(self.t.ndm)) if dms is None else list(dms)
        res: list[np.ndarray] = []
        self.search_ms = []
        for i, d in enumerate(dms):
            ses = self.sessions[i & 1]
            # ses's previous search (DM i-2) was collected in iteration i-1
            self._spectrum(d, ses)
            ses.enqueue(None, threshold, after_stream=self.stream.cuda_stream)
            if i > 0:
                res.append(self._finish(self.sessions[(i - 1) & 1], threshold, collapse))
        if dms:
            res.append(self._finish(self.sessions[(len(dms) - 1) & 1], threshold, collapse))
        return res

    def run(self, d_raw: int, nspec: int, collapse: bool = True) -> list[np.ndarray]:
        """Candidates of every DM, in DM order (collapsed as search_file does
        unless collapse is False)."""
        self.dedisperse(d_raw, nspec)
        return self.search_all(collapse=collapse)

    def series(self, d: int) -> np.ndarray:
        self.stream.synchronize()
        return self.out[d, :self.N].cpu().numpy()

    def close(self) -> None:
        for ses in getattr(self, "sessions", []) or []:
            ses.close()
        self.sessions = []
        self.ses = None
        for name in ("spec", "dd"):
            obj = getattr(self, name, None)
            if obj is not None:
                obj.close()
                setattr(self, name, None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
