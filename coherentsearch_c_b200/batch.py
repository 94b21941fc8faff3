"""Batched search of many spectra through cs_gpu_batch_* (libcsgpu.so).

    with Batch(nslots=3) as b:
        ids = [b.submit(amps_i, N_i, dt, Options(nharms=60)) for ...]
        for i in ids:
            raw, queued_ms, run_ms = b.wait(i)

Each result is exactly what Session.run_raw (cs_gpu_session_run) returns for
the same spectrum and options: the raw, uncollapsed candidates.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as nt
from .search import Options, _as_amps, _file


class BatchCancelled(RuntimeError):
    """The request was cancelled before a slot took it."""


class Batch:
    """A pool of search slots on one GPU (cs_gpu_batch_create)."""

    def __init__(self, device: int = 0, nslots: int = 3, mem_budget: int = 0):
        self.gpu = nt.gpu_lib()
        self.host = nt.host_lib()
        self.h = self.gpu.cs_gpu_batch_create(device, nslots, int(mem_budget))
        if not self.h:
            raise RuntimeError("cs_gpu_batch_create failed (see stderr)")
        self._keep: dict[int, tuple] = {}

    def submit(self, amps, N: int, dt: float, opts: Options | None = None) -> int:
        """Queue one spectrum (complex64[N/2] or interleaved float32); returns its id."""
        opts = opts or Options()
        a = _as_amps(amps)
        if a.size != 2 * (N // 2):
            raise ValueError("spectrum length does not match N")
        ft = _file(a, N, dt)
        p = opts.params(self.host)
        rid = self.gpu.cs_gpu_batch_submit(self.h, C.byref(ft), C.byref(p), opts.lofreq,
                                           opts.hifreq, opts.lobin, opts.blocksize,
                                           opts.threshold)
        if rid < 0:
            raise RuntimeError("cs_gpu_batch_submit failed")
        self._keep[rid] = (a, ft, p)          # the spectrum must outlive the request
        return rid

    def wait(self, rid: int) -> tuple[np.ndarray, float, float]:
        """(raw candidates, ms queued for a slot, ms on the slot)."""
        cl = nt.CandidateList()
        q, r = C.c_double(0), C.c_double(0)
        rc = self.gpu.cs_gpu_batch_wait(self.h, rid, C.byref(cl), C.byref(q), C.byref(r))
        self._keep.pop(rid, None)
        out = nt.candidates_to_numpy(cl)
        self.host.candlist_free(C.byref(cl))
        if rc == -2:
            raise BatchCancelled(f"batch request {rid} was cancelled")
        if rc != 0:
            raise RuntimeError(f"batch request {rid} failed (see stderr)")
        return out, q.value, r.value

    def cancel(self, rid: int) -> bool:
        """Drop a request no slot has taken yet (its wait then raises
        BatchCancelled); False if it is already running or finished."""
        rc = self.gpu.cs_gpu_batch_cancel(self.h, rid)
        if rc < 0:
            raise KeyError(rid)
        return rc == 0

    def warm(self, N: int, dt: float, opts: Options | None = None) -> None:
        """Load every slot for a length-N search with `opts` (no spectrum is
        read), so that requests up to that size find their buffers grown."""
        opts = opts or Options()
        ft = nt.FFTFile()
        ft.amps = None
        ft.namps = N // 2
        ft.N = N
        ft.T = N * dt
        ft.df = 1.0 / ft.T
        p = opts.params(self.host)
        if self.gpu.cs_gpu_batch_warm(self.h, C.byref(ft), C.byref(p), opts.lofreq, opts.hifreq,
                                      opts.lobin, opts.blocksize) != 0:
            raise RuntimeError("cs_gpu_batch_warm failed (see stderr)")

    def device_bytes(self) -> int:
        """Device memory the slots hold now (what admission keeps within
        the budget)."""
        return int(self.gpu.cs_gpu_batch_device_bytes(self.h))

    def pending(self) -> int:
        return int(self.gpu.cs_gpu_batch_pending(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.gpu.cs_gpu_batch_free(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
