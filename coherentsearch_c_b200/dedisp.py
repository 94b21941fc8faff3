"""Subband dedispersion of 8-bit filterbank data (prepsubband's stage of the
reference raw-data front end) through libcsgpu.so's cs_dedisp_* ABI.

    tables = dedisp_tables(nchan=1024, nsub=64, ndm=500, lodm=0.0, dmstep=0.4,
                           lofreq=1250.146484375, chanwid=300/1024, dt=64e-6)
    with Dedisperser(tables, max_spectra=raw.shape[0]) as dd:
        out = dd.run(raw)            # [ndm][nout] float32

`raw` is [nspec][nchan] uint8 in SIGPROC order (highest frequency first).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native as nt

SPECTRA_PER_SUBINT = 2400     # SIGPROC reader block (third_party/presto/src/sigproc_fb.c:422)


@dataclass
class DedispTables:
    nchan: int
    nsub: int
    ndm: int
    idispdt: np.ndarray       # [nchan] int32, ascending frequency
    offsets: np.ndarray       # [ndm, nsub] int32
    blocks_per_read: int
    avgdm: float
    spectra_per_subint: int = SPECTRA_PER_SUBINT


def dedisp_tables(nchan: int, nsub: int, ndm: int, lodm: float, dmstep: float, lofreq: float,
                  chanwid: float, dt: float,
                  spectra_per_subint: int = SPECTRA_PER_SUBINT) -> DedispTables:
    """Delay tables exactly as src/prep_dedisp.c builds them (cs_dedisp_tables)."""
    lib = nt.gpu_lib()
    idisp = np.zeros(nchan, np.int32)
    offs = np.zeros((ndm, nsub), np.int32)
    bpr = C.c_int(0)
    avg = C.c_double(0)
    ip = C.POINTER(C.c_int)
    rc = lib.cs_dedisp_tables(nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt,
                              spectra_per_subint, idisp.ctypes.data_as(ip),
                              offs.ctypes.data_as(ip), C.byref(bpr), C.byref(avg))
    if rc != 0:
        raise ValueError("cs_dedisp_tables rejected the geometry")
    return DedispTables(nchan, nsub, ndm, idisp, offs, bpr.value, avg.value, spectra_per_subint)


def output_length(tables: DedispTables, nspec: int, numout: int = -1) -> int:
    """Points per DM the reference writes: whole output chunks only
    (src/prep_dedisp.c:484-522), at most numout."""
    L, bpr = tables.spectra_per_subint, tables.blocks_per_read
    nb = nspec // L
    k = max((nb - 1) // bpr - 1, 0) if nb >= 1 else 0
    n = k * L * bpr
    return min(n, numout) if numout >= 0 else n


class Dedisperser:
    """A cs_dedisp plan on one GPU."""

    def __init__(self, tables: DedispTables, max_spectra: int, device: int = 0):
        self.t = tables
        self.device = device
        self.lib = nt.gpu_lib()
        ip = C.POINTER(C.c_int)
        self._idisp = np.ascontiguousarray(tables.idispdt, np.int32)
        self._offs = np.ascontiguousarray(tables.offsets, np.int32)
        self.plan = self.lib.cs_dedisp_create(
            tables.nchan, tables.nsub, tables.ndm, self._idisp.ctypes.data_as(ip),
            self._offs.ctypes.data_as(ip), tables.spectra_per_subint, tables.blocks_per_read,
            int(max_spectra), device)
        if not self.plan:
            raise RuntimeError("cs_dedisp_create failed (see stderr)")

    def output_length(self, nspec: int, numout: int = -1) -> int:
        return int(self.lib.cs_dedisp_output_length(self.plan, nspec, numout))

    def run(self, raw: np.ndarray, numout: int = -1) -> np.ndarray:
        """Host arrays in and out (cs_dedisp_run)."""
        raw = np.ascontiguousarray(raw, np.uint8)
        if raw.ndim != 2 or raw.shape[1] != self.t.nchan:
            raise ValueError("raw must be [nspec][nchan] uint8")
        n = self.output_length(raw.shape[0], numout)
        out = np.zeros((self.t.ndm, max(n, 1)), np.float32)
        got = C.c_longlong(0)
        rc = self.lib.cs_dedisp_run(self.plan, raw.ctypes.data, raw.shape[0], numout,
                                    out.ctypes.data, out.shape[1], C.byref(got))
        if rc != 0:
            raise RuntimeError("cs_dedisp_run failed (see stderr)")
        return out[:, :got.value]

    def run_device(self, d_raw: int, nspec: int, d_out: int, out_stride: int,
                   numout: int = -1, stream: int | None = None) -> int:
        """Device pointers (cs_dedisp_run_device); returns points per DM.
        stream: a cudaStream_t handle; None or 0 selects the plan's stream."""
        got = C.c_longlong(0)
        rc = self.lib.cs_dedisp_run_device(self.plan, d_raw, nspec, numout, d_out, out_stride,
                                           stream, C.byref(got))
        if rc != 0:
            raise RuntimeError("cs_dedisp_run_device failed (see stderr)")
        return got.value

    def run_device_clipped(self, d_raw: int, nspec: int, d_flags: int, d_levels: int,
                           d_out: int, out_stride: int, numout: int = -1,
                           stream: int | None = None) -> int:
        """cs_dedisp_run_device_clipped: the run prepsubband makes with -clip,
        given clip_levels' flags and levels (device pointers); returns points
        per DM.  The first clipped run allocates the plan's float subbands."""
        got = C.c_longlong(0)
        rc = self.lib.cs_dedisp_run_device_clipped(self.plan, d_raw, nspec, numout, d_flags,
                                                   d_levels, d_out, out_stride, stream,
                                                   C.byref(got))
        if rc != 0:
            raise RuntimeError("cs_dedisp_run_device_clipped failed (see stderr)")
        return got.value

    def clip_levels(self, d_raw: int, nspec: int, d_flags: int, d_levels: int,
                    clip_sigma: float = 6.0, stream: int | None = None,
                    scratch: int | None = None, scratch_bytes: int = 0) -> int:
        """cs_clip_levels: the count of replaced spectra, their flags
        (nspec // L * L bytes at d_flags) and clip_times' channel levels after
        each block ([nspec // L][nchan] floats at d_levels, SIGPROC channel
        order)."""
        n = C.c_longlong(0)
        rc = self.lib.cs_clip_levels(d_raw, nspec, self.t.nchan, self.t.spectra_per_subint,
                                     float(clip_sigma), C.byref(n), d_flags, d_levels, scratch,
                                     scratch_bytes, stream, self.device)
        if rc != 0:
            raise RuntimeError("cs_clip_levels failed (see stderr)")
        return n.value

    def clip_scratch_bytes(self, nspec: int) -> int:
        return int(self.lib.cs_clip_scratch_bytes(nspec, self.t.spectra_per_subint))

    def clip_count(self, d_raw: int, nspec: int, clip_sigma: float = 6.0,
                   stream: int | None = None, scratch: int | None = None,
                   scratch_bytes: int = 0) -> int:
        """cs_clip_count: the spectra prepsubband's -clip clip_sigma would
        replace in this filterbank (0: the unclipped output is the clipped
        run's).  scratch: a device buffer of clip_scratch_bytes(nspec) bytes
        kept across calls (None: the call allocates its own)."""
        n = C.c_longlong(0)
        rc = self.lib.cs_clip_count(d_raw, nspec, self.t.nchan, self.t.spectra_per_subint,
                                    float(clip_sigma), C.byref(n), None, scratch,
                                    scratch_bytes, stream, self.device)
        if rc != 0:
            raise RuntimeError("cs_clip_count failed (see stderr)")
        return n.value

    def last_times(self) -> tuple[float, float]:
        a, b = C.c_float(0), C.c_float(0)
        if self.lib.cs_dedisp_last_times(self.plan, C.byref(a), C.byref(b)) != 0:
            raise RuntimeError("cs_dedisp_last_times failed")
        return a.value, b.value

    def close(self) -> None:
        if getattr(self, "plan", None):
            self.lib.cs_dedisp_free(self.plan)
            self.plan = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
