"""Python mirror of the reference search interface.

`search_spectrum` is search_file() (src/search.c:1247) on an in-memory
spectrum; `Session` holds the plan cache and one GPU session
(cs_gpu_session_create / run, src/cuda.cu:554-1176) for repeated searches of
spectra with the same geometry, and exposes the device-resident path used for
timing.  All compute runs in libcsgpu.so; there is no CPU fallback: if the
extension or the GPU is missing, these calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import native as nt


@dataclass
class Options:
    """Search options with the reference CLI defaults (src/cli.c:351-381)."""
    nharms: int = 60
    m: int = 16
    hidr: float = 0.5
    threshold: float = 8.0
    lobin: int = 100
    lofreq: float = 0.1
    hifreq: float = 125.0
    blocksize: int = 65536          # GPU default (src/cli.c:920)
    maxdecim: int = 6
    drtol: float = 1.0
    numharm: int = 16
    remove: bool = True
    harm_remove: bool = True
    boxcar_fsp: float = 1.5
    boxcar_maxfrac: float = 0.3
    precision: int = 0              # 0: f32, 1: f64 (--precision, CS_PREC_F64)

    def params(self, lib) -> nt.SearchParams:
        p = nt.SearchParams()
        lib.params_defaults(C.byref(p))
        p.nharms = self.nharms
        p.m = self.m
        p.hidr = self.hidr
        p.threshold = self.threshold
        p.boxcar_fsp = self.boxcar_fsp
        p.boxcar_maxfrac = self.boxcar_maxfrac
        p.ndecim = lib.decimation_set(self.nharms, self.maxdecim, p.decimations, 64)
        p.precision = self.precision
        return p

    def geometry(self, N: int, dt: float):
        """(r_lo, lodr, total) exactly as src/search.c:1257-1264."""
        T = N * dt
        lodr = self.hidr / float(self.nharms)
        r_lo = self.lofreq * T
        if self.lobin != 100:
            r_lo = float(self.lobin)
        r_hi = self.hifreq * T
        total = int(math.floor((r_hi - r_lo) / lodr)) + 1
        return r_lo, lodr, max(total, 0)


_libc_free = C.CDLL(None).free
_libc_free.argtypes = [C.c_void_p]
_libc_free.restype = None


def _as_amps(amps) -> np.ndarray:
    a = np.ascontiguousarray(amps)
    if a.dtype == np.complex64:
        a = a.view(np.float32)
    if a.dtype != np.float32:
        raise TypeError("amps must be complex64[namps] or float32[2*namps]")
    return a


def _file(amps: np.ndarray, N: int, dt: float) -> nt.FFTFile:
    ft = nt.FFTFile()
    ft.amps = amps.ctypes.data_as(C.POINTER(C.c_float))
    ft.namps = amps.size // 2
    ft.N = N
    ft.T = N * dt
    ft.df = 1.0 / ft.T
    ft.inf.N = N
    ft.inf.has_N = 1
    ft.inf.dt = dt
    ft.inf.has_dt = 1
    return ft


def gpu_available(device: int = 0) -> tuple[int, str]:
    buf = C.create_string_buffer(256)
    rc = nt.gpu_lib().cs_gpu_available(device, buf, 256)
    return rc, buf.value.decode()


def search_spectrum(amps, N: int, dt: float, opts: Options | None = None,
                    device: int = 0, ducy: bool = False) -> np.ndarray:
    """search_file() on a PRESTO-packed spectrum (namps = N/2 complex, bin 0
    = (DC, Nyquist)).  Returns the collapsed candidates (CAND_DTYPE)."""
    opts = opts or Options()
    lib = nt.host_lib()
    a = _as_amps(amps)
    ft = _file(a, N, dt)
    p = opts.params(lib)
    cl = lib.search_file(C.byref(ft), C.byref(p), opts.lofreq, opts.hifreq, opts.lobin,
                         opts.blocksize, opts.threshold, int(opts.remove), opts.drtol,
                         int(opts.harm_remove), opts.numharm, None, 0, 0, 0, None, None,
                         1.0, device)
    if ducy:
        cl2 = lib.measure_ducy(C.byref(ft), C.byref(cl), C.byref(p))
        lib.candlist_free(C.byref(cl))
        cl = cl2
    out = nt.candidates_to_numpy(cl)
    lib.candlist_free(C.byref(cl))
    return out


class Session:
    """Plans + one GPU session for spectra of a fixed geometry (N, dt, options)."""

    def __init__(self, N: int, dt: float, opts: Options | None = None, device: int = 0):
        self.opts = opts or Options()
        self.N, self.dt, self.device = N, dt, device
        self.host = nt.host_lib()
        self.gpu = nt.gpu_lib()
        self.params = self.opts.params(self.host)
        self.r_lo, self.lodr, self.total = self.opts.geometry(N, dt)
        if self.total <= 0:
            raise ValueError("empty trial range")
        self.namps = N // 2
        # planning reads the geometry only (N, namps, T), never the amplitudes
        self._dummy = np.zeros(2, dtype=np.float32)
        self.ft = _file(self._dummy, N, dt)
        self.ft.namps = self.namps
        self.plans = nt.DirectPlanSet()
        if self.host.direct_plans_build(C.byref(self.plans), C.byref(self.params), self.r_lo):
            raise RuntimeError("direct_plans_build failed")
        cs = C.POINTER(C.c_longlong)()
        nch = C.c_longlong(0)
        if self.host.chunk_starts(C.byref(self.plans), C.byref(self.ft), C.byref(self.params),
                                  self.total, self.opts.blocksize, C.byref(cs), C.byref(nch)):
            raise RuntimeError("chunk_starts failed")
        self.nchunks = nch.value
        self.cstarts = np.ctypeslib.as_array(cs, shape=(self.nchunks,)).copy()
        _libc_free(cs)
        self._cs = self.cstarts.ctypes.data_as(C.POINTER(C.c_longlong))
        self.sess = self.gpu.cs_gpu_session_create(
            C.byref(self.ft), C.byref(self.params), C.byref(self.plans), self._cs, self.total,
            self.opts.blocksize, self.nchunks, self.r_lo, self.lodr, device)
        if not self.sess:
            raise RuntimeError("cs_gpu_session_create failed (see stderr)")

    def info(self) -> nt.CsB200Info:
        inf = nt.CsB200Info()
        self.gpu.cs_b200_session_info(self.sess, C.byref(inf))
        return inf

    def run_raw(self, amps, threshold: float | None = None) -> np.ndarray:
        """cs_gpu_session_run: uncollapsed candidates in the reference order."""
        a = _as_amps(amps)
        if a.size != 2 * self.namps:
            raise ValueError("spectrum length does not match the session")
        ft = _file(a, self.N, self.dt)
        thr = self.opts.threshold if threshold is None else threshold
        cl = self.gpu.cs_gpu_session_run(self.sess, C.byref(ft), thr)
        out = nt.candidates_to_numpy(cl)
        self.host.candlist_free(C.byref(cl))
        return out

    def collapse(self, raw: np.ndarray) -> np.ndarray:
        """The post-processing of search_file (src/search.c:1467-1478) on the
        host: remove_duplicates when `remove`, else a stable frequency sort;
        then remove_harmonics when `harm_remove`."""
        if self.opts.remove:
            n = raw.size
            buf = (nt.Candidate * max(n, 1))()
            if n:
                C.memmove(buf, raw.ctypes.data, n * C.sizeof(nt.Candidate))
            cl = nt.CandidateList(C.cast(buf, C.POINTER(nt.Candidate)), n, n)
            cl = self.host.remove_duplicates(C.byref(cl), self.opts.drtol)
            arr = nt.candidates_to_numpy(cl)
            self.host.candlist_free(C.byref(cl))
        else:
            arr = raw[np.argsort(raw["freq"], kind="stable")]
        if self.opts.harm_remove:
            n = arr.size
            buf = (nt.Candidate * max(n, 1))()
            if n:
                C.memmove(buf, np.ascontiguousarray(arr).ctypes.data, n * C.sizeof(nt.Candidate))
            cl = nt.CandidateList(C.cast(buf, C.POINTER(nt.Candidate)), n, n)
            cl2 = self.host.remove_harmonics(C.byref(cl), self.opts.numharm, 1.0)
            arr = nt.candidates_to_numpy(cl2)
            self.host.candlist_free(C.byref(cl2))
        return arr

    def collect_collapsed(self, threshold: float | None = None):
        """cs_b200_session_collect_collapsed: the enqueued search's candidates
        harvested and collapsed on the GPU (the records stay on the device).
        Returns (candidates, kernel ms, rc) like collect."""
        thr = self.opts.threshold if threshold is None else threshold
        cl = nt.CandidateList()
        ms = C.c_float(0)
        o = self.opts
        rc = self.gpu.cs_b200_session_collect_collapsed(self.sess, thr, int(o.remove), o.drtol,
                                                        int(o.harm_remove), o.numharm, 1.0,
                                                        C.byref(cl), C.byref(ms))
        if rc < 0:
            raise RuntimeError("collect_collapsed failed")
        out = nt.candidates_to_numpy(cl)
        self.host.candlist_free(C.byref(cl))
        return out, ms.value, rc

    def collapse_enqueue(self, threshold: float | None = None) -> int:
        """First half of collect_collapsed: waits for the search, queues the
        collapse; returns 0, or 1 when the record buffer was grown (enqueue
        the search again)."""
        thr = self.opts.threshold if threshold is None else threshold
        o = self.opts
        rc = self.gpu.cs_b200_session_collapse_enqueue(self.sess, thr, int(o.remove), o.drtol,
                                                       int(o.harm_remove), o.numharm, 1.0)
        if rc < 0:
            raise RuntimeError("collapse_enqueue failed")
        return rc

    def collapse_wait(self):
        """Second half: (candidates, kernel ms)."""
        cl = nt.CandidateList()
        ms = C.c_float(0)
        if self.gpu.cs_b200_session_collapse_wait(self.sess, C.byref(cl), C.byref(ms)) != 0:
            raise RuntimeError("collapse_wait failed")
        out = nt.candidates_to_numpy(cl)
        self.host.candlist_free(C.byref(cl))
        return out, ms.value

    def measure_ducy(self, cands: np.ndarray) -> np.ndarray:
        """measure_ducy (src/candidate.c:305-329) on the GPU against the
        spectrum this session last searched (still in device memory): a copy
        of `cands` with the ducy field filled in."""
        out = np.array(cands, dtype=nt.CAND_DTYPE, copy=True)
        if out.size == 0:
            return out
        if getattr(self, "_ducy", None) is None:
            self._ducy = self.gpu.cs_ducy_create(self.params.boxcar_fsp,
                                                  self.params.boxcar_maxfrac, self.device)
            if not self._ducy:
                raise RuntimeError("cs_ducy_create failed (see stderr)")
        d = np.empty(out.size, dtype=np.float64)
        rc = self.gpu.cs_ducy_run_device(self._ducy, self.device_amps_ptr(), self.namps, self.N,
                                         out.ctypes.data, out.size,
                                         d.ctypes.data_as(C.POINTER(C.c_double)), None)
        if rc != 0:
            raise RuntimeError("cs_ducy_run_device failed (see stderr)")
        out["ducy"] = d
        return out

    def device_amps_ptr(self) -> int:
        return int(self.gpu.cs_b200_session_device_amps(self.sess))

    def enqueue(self, d_amps_ptr: int | None = None, threshold: float | None = None,
                after_stream: int | None = None) -> None:
        """Queue a search; with `after_stream` (a cudaStream_t handle) it
        starts after the work already queued there (the spectrum's producer)."""
        thr = self.opts.threshold if threshold is None else threshold
        rc = self.gpu.cs_b200_session_enqueue_device(self.sess, d_amps_ptr, thr,
                                                     after_stream or None)
        if rc != 0:
            raise RuntimeError("enqueue failed")

    def collect(self, threshold: float | None = None):
        thr = self.opts.threshold if threshold is None else threshold
        cl = nt.CandidateList()
        ms = C.c_float(0)
        rc = self.gpu.cs_b200_session_collect(self.sess, thr, C.byref(cl), C.byref(ms))
        if rc < 0:
            raise RuntimeError("collect failed")
        out = nt.candidates_to_numpy(cl)
        self.host.candlist_free(C.byref(cl))
        return out, ms.value, rc

    def close(self) -> None:
        if getattr(self, "_ducy", None):
            self.gpu.cs_ducy_free(self._ducy)
            self._ducy = None
        if getattr(self, "sess", None):
            self.gpu.cs_gpu_session_free(self.sess)
            self.sess = None
        if getattr(self, "plans", None) is not None and self.plans.n:
            self.host.direct_plans_free(C.byref(self.plans))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def multi_enqueue(sessions, d_amps=None, threshold: float | None = None, stream=None) -> None:
    """Queue one persistent launch over the tiles of several spectra
    (cs_b200_multi_enqueue).  The sessions must share one warp-specialised
    configuration (nharms, ladder).  d_amps: device spectrum pointers (None:
    each session's own buffer); stream: a cudaStream_t handle the launch
    follows (None: the first session's stream)."""
    gpu = nt.gpu_lib()
    n = len(sessions)
    thr = sessions[0].opts.threshold if threshold is None else threshold
    arr = (C.c_void_p * n)(*[s.sess for s in sessions])
    amps = None
    if d_amps is not None:
        amps = (C.c_void_p * n)(*[int(p) if p else None for p in d_amps])
    if gpu.cs_b200_multi_enqueue(arr, n, amps, thr, stream) != 0:
        raise RuntimeError("cs_b200_multi_enqueue failed")


def multi_collect(sessions, d_amps=None, threshold: float | None = None):
    """Each session's raw candidates after multi_enqueue (a session whose
    record buffer overflowed is searched again on its own)."""
    thr = sessions[0].opts.threshold if threshold is None else threshold
    outs, kms = [], 0.0
    for i, s in enumerate(sessions):
        out, ms, rc = s.collect(thr)
        if i == 0:
            kms = ms
        if rc == 1:
            s.enqueue(d_amps[i] if d_amps is not None else None, thr)
            out, _, rc = s.collect(thr)
        outs.append(out)
    return outs, kms


def multi_search(sessions, d_amps=None, threshold: float | None = None, stream=None):
    """multi_enqueue then multi_collect: (list of candidate arrays, kernel ms)."""
    if not sessions:
        return [], 0.0
    multi_enqueue(sessions, d_amps, threshold, stream)
    return multi_collect(sessions, d_amps, threshold)


class MultiGraph:
    """A multi-spectrum search recorded once as a CUDA graph
    (cs_b200_multi_graph_create) and replayed with launch(); collect() gives
    each session's raw candidates, as multi_collect does after
    multi_enqueue.  The graph holds the sessions' buffer addresses: close it
    before the sessions, and build a new one after a session is reloaded or
    grows its record buffer (launch raises StaleGraph then)."""

    class StaleGraph(RuntimeError):
        pass

    def __init__(self, sessions, d_amps=None, threshold: float | None = None):
        self.gpu = nt.gpu_lib()
        self.sessions = list(sessions)
        self.d_amps = d_amps
        self.threshold = self.sessions[0].opts.threshold if threshold is None else threshold
        n = len(self.sessions)
        arr = (C.c_void_p * n)(*[s.sess for s in self.sessions])
        amps = None
        if d_amps is not None:
            amps = (C.c_void_p * n)(*[int(p) if p else None for p in d_amps])
        self.graph = self.gpu.cs_b200_multi_graph_create(arr, n, amps, self.threshold)
        if not self.graph:
            raise RuntimeError("cs_b200_multi_graph_create failed")

    def launch(self, stream=None) -> None:
        rc = self.gpu.cs_b200_multi_graph_launch(self.graph, stream)
        if rc == -2:
            raise MultiGraph.StaleGraph("a session changed since the capture")
        if rc != 0:
            raise RuntimeError("cs_b200_multi_graph_launch failed")

    def collect(self):
        return multi_collect(self.sessions, self.d_amps, self.threshold)

    def search(self, stream=None):
        self.launch(stream)
        return self.collect()

    def close(self) -> None:
        if getattr(self, "graph", None):
            self.gpu.cs_b200_multi_graph_free(self.graph)
            self.graph = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
