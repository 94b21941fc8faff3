"""The raw-data front end on one GPU: 8-bit filterbank -> subband
dedispersion -> for every DM, the series padded to `numout` points ->
realfft + rednoise -> coherent search, as the reference's
prep_coherent_search runs it (src/prep_dedisp.c:484-522, 744-790;
src/prep_search.c), with prepsubband's time-domain clipping (-clip, 6 sigma
by default) and without masking, downsampling or barycentring.

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

    Four search sessions of the one geometry take the DMs in turn.  At DM i
    the host queues DM i's spectrum (prep stream) and search, then DM i-2's
    collapse (which first waits for DM i-2's search), then takes DM i-3's
    list, so two searches stay queued ahead of the host and a host stall of a
    few milliseconds does not idle the GPU.  Without collapsing, DM i-1's raw
    records are read back while DM i is searched."""

    def __init__(self, tables: DedispTables, nspec: int, numout: int, dt: float,
                 opts: Options | None = None, device: int = 0, clip_sigma: float = 6.0):
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
        self.sessions = [Session(self.N, dt, self.opts, device=device) for _ in range(4)]
        self.ses = self.sessions[0]
        self.pad_value = None
        # prepsubband clips at 6 sigma unless told -noclip (0 here)
        self.clip_sigma = float(clip_sigma)
        self.nclipped = 0                    # spectra the last dedisperse replaced
        self.search_ms: list[float] = []     # search kernel time of each DM, last pass

    def dedisperse(self, d_raw: int, nspec: int) -> None:
        """Dedisperse [nspec][nchan] uint8 at device address d_raw, then pad
        every series from nout to N with DM 0's running mean."""
        torch = self.torch
        # the raw block may still be in flight on the caller's stream
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))
        self.nclipped = 0
        if self.clip_sigma > 0:
            L = self.t.spectra_per_subint
            nblk = nspec // L
            # kept across calls: allocating here would synchronise the device
            self._clip_scratch = self._keep("_clip_scratch", self.dd.clip_scratch_bytes(nspec),
                                            torch.uint8)
            self._clip_flags = self._keep("_clip_flags", nblk * L, torch.uint8)
            self._clip_levels = self._keep("_clip_levels", nblk * self.t.nchan, torch.float32)
            self.nclipped = self.dd.clip_levels(
                d_raw, nspec, self._clip_flags.data_ptr(), self._clip_levels.data_ptr(),
                self.clip_sigma, self.stream.cuda_stream, self._clip_scratch.data_ptr(),
                self._clip_scratch.numel())
        if self.nclipped:
            n = self.dd.run_device_clipped(d_raw, nspec, self._clip_flags.data_ptr(),
                                           self._clip_levels.data_ptr(), self.out.data_ptr(),
                                           self.stride, self.N, self.stream.cuda_stream)
        else:
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

    def _keep(self, name: str, n: int, dtype):
        """A device buffer of at least n elements, grown only when too small."""
        buf = getattr(self, name, None)
        if buf is None or buf.numel() < n:
            buf = self.torch.empty(max(1, n), dtype=dtype, device=self.dev)
        return buf

    def _spectrum(self, d: int, ses: Session) -> None:
        self.spec.run_device(self.out[d].data_ptr(), ses.device_amps_ptr(),
                             self.stream.cuda_stream)

    def search_dm(self, d: int, threshold: float | None = None) -> np.ndarray:
        """Spectrum and search of DM d's series: raw candidates."""
        ses = self.sessions[0]
        self._spectrum(d, ses)
        ses.enqueue(None, threshold, after_stream=self.stream.cuda_stream)
        out, _, rc = ses.collect(threshold)
        if rc == 1:                     # record buffer grown: run again
            ses.enqueue(None, threshold)
            out, _, rc = ses.collect(threshold)
        return out

    def search_all(self, threshold: float | None = None, dms=None,
                   collapse: bool = False) -> list[np.ndarray]:
        """Candidates of every DM (or of `dms`) in DM order: raw, or with
        `collapse` the list search_file returns, collapsed on the GPU."""
        dms = list(range(self.t.ndm)) if dms is None else list(dms)
        self.search_ms = [0.0] * len(dms)
        S, ns = self.sessions, len(self.sessions)
        res: list = [None] * len(dms)

        def start_collapse(j: int) -> None:
            ses = S[j % ns]
            while ses.collapse_enqueue(threshold) == 1:   # record buffer grown
                ses.enqueue(None, threshold)

        def finish(j: int) -> None:
            if collapse:
                res[j], self.search_ms[j] = S[j % ns].collapse_wait()
            else:
                ses = S[j % ns]
                out, ms, rc = ses.collect(threshold)
                if rc == 1:
                    ses.enqueue(None, threshold)
                    out, ms, rc = ses.collect(threshold)
                res[j], self.search_ms[j] = out, ms

        for i, d in enumerate(dms):
            ses = S[i % ns]          # its last DM, i - ns, was finished at i - 1
            self._spectrum(d, ses)
            ses.enqueue(None, threshold, after_stream=self.stream.cuda_stream)
            if collapse:
                if i >= 2:
                    start_collapse(i - 2)
                if i >= 3:
                    finish(i - 3)
            elif i >= 1:
                finish(i - 1)
        n = len(dms)
        if collapse:
            for j in range(max(0, n - 2), n):
                start_collapse(j)
            for j in range(max(0, n - 3), n):
                finish(j)
        elif n >= 1:
            finish(n - 1)
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
