"""Test-side bindings of the checkers under oracle/:

* libcsref.so     -- the reference's own CPU search path (src/*.c compiled
                     unmodified by oracle/Makefile against the FFTW-API shim)
* libcsoracle.so  -- oracle/cs_oracle.c, the per-trial CPU restatement
* libdedisp_ref.so -- the reference's vendored PRESTO dispersion.c
* libcsref_gpu.so  -- the reference's search path on its own src/cuda.cu
                     backend for sm_100a (the plain GPU form)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from coherentsearch_c_b200 import native as nt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

_REF = None
_ORA = None


def have_ref() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libcsref.so"))


def pin_ref_threads(n: int = 1) -> None:
    """Run the reference's OpenMP chunk loop (src/search.c:1044-1055) on n
    threads of the calling thread's team.

    The reference is deterministic only on one thread: each thread's
    workspace caches a decimated slot's boxcar normalisation and refreshes it
    when the NUMBER of filled harmonics changes (src/search.c:36-45), while
    the normalisation depends on WHICH harmonics are filled
    (src/boxcar.c:170-195).  With chunks dealt round-robin, a thread can go
    from a low-band chunk (low harmonics missing) to a high-band chunk (top
    harmonics missing) with the same count and keep the stale shape; with 16
    threads on a 24576-point, 128 us spectrum this adds 13 candidates in one
    chunk of the k=3 slot.  On one thread the chunks run in r order and the
    cache is always current, which is the search's intended result."""
    C.CDLL("libgomp.so.1").omp_set_num_threads(int(n))


def ref_lib() -> C.CDLL:
    global _REF
    if _REF is None:
        pin_ref_threads(1)
        # CS_REF_LIBNAME=libcsref_timed.so loads the build whose FFT shim
        # counts the time spent in its transforms (cs_shim_fft_seconds)
        name = os.environ.get("CS_REF_LIBNAME", "libcsref.so")
        lib = nt.declare_host_api(C.CDLL(os.path.join(REF_DIR, name)))
        lib.datpipe_create.argtypes = [C.c_int, C.c_int, C.c_double]
        lib.datpipe_create.restype = C.c_void_p
        lib.datpipe_free.argtypes = [C.c_void_p]
        lib.datpipe_redfft_mem.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_longlong,
                                           C.c_double, C.c_char_p, C.POINTER(nt.FFTFile)]
        lib.datpipe_redfft_mem.restype = C.c_int
        lib.search_cache_free.argtypes = [C.c_void_p]
        _REF = lib
    return _REF


def have_ref_gpu() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libcsref_gpu.so"))


_REF_GPU = None


def ref_gpu_lib() -> C.CDLL:
    """The reference's search path with its own src/cuda.cu backend (the
    plain single-file GPU form), built by `make -C oracle refgpu`."""
    global _REF_GPU
    if _REF_GPU is None:
        ref_lib()                       # pins the OpenMP team before the load
        _REF_GPU = nt.declare_host_api(C.CDLL(os.path.join(REF_DIR, "libcsref_gpu.so")))
    return _REF_GPU


def ref_search_gpu(amps: np.ndarray, N: int, dt: float, opts, device: int = 0,
                   collapse: bool = True) -> np.ndarray:
    """The reference's search_file (src/search.c:1247) on its own GPU backend
    (src/search.c:1374-1406 -> src/cuda.cu), one session per call."""
    lib = ref_gpu_lib()
    ft = make_file(amps, N, dt)
    p = opts.params(lib)
    rem = int(opts.remove) if collapse else 0
    hrem = int(opts.harm_remove) if collapse else 0
    cl = lib.search_file(C.byref(ft), C.byref(p), opts.lofreq, opts.hifreq, opts.lobin,
                         opts.blocksize, opts.threshold, rem, opts.drtol, hrem, opts.numharm,
                         None, 0, 0, 0, None, None, 1.0, int(device))
    out = nt.candidates_to_numpy(cl)
    lib.candlist_free(C.byref(cl))
    return out


class RefGpuSearcher:
    """The reference's GPU form with its SearchCache kept across calls (the
    session is reused while the geometry matches, src/search.c:1388-1406), as
    its list driver runs a sweep of equal-length files (src/cli.c:976)."""

    def __init__(self, opts, device: int = 0):
        self.lib = ref_gpu_lib()
        self.lib.search_cache_free.argtypes = [C.c_void_p]
        self.opts = opts
        self.device = device
        self.p = opts.params(self.lib)           # one address: part of the session match
        self.cache = C.create_string_buffer(8192)  # zeroed, as the CLI memsets it

    def search(self, amps: np.ndarray, N: int, dt: float, collapse: bool = True):
        o = self.opts
        ft = make_file(amps, N, dt)
        cl = self.lib.search_file(C.byref(ft), C.byref(self.p), o.lofreq, o.hifreq, o.lobin,
                                  o.blocksize, o.threshold, int(o.remove) if collapse else 0,
                                  o.drtol, int(o.harm_remove) if collapse else 0, o.numharm,
                                  None, 0, 0, 0, None, C.addressof(self.cache), 1.0,
                                  int(self.device))
        out = nt.candidates_to_numpy(cl)
        self.lib.candlist_free(C.byref(cl))
        return out

    def close(self) -> None:
        if self.cache is not None:
            self.lib.search_cache_free(C.addressof(self.cache))
            self.cache = None


def oracle_lib() -> C.CDLL:
    global _ORA
    if _ORA is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libcsoracle.so"))
        lib.cso_trial_metrics.argtypes = [
            C.POINTER(C.c_float), C.c_longlong, C.c_longlong, C.c_int, C.c_int, C.c_double,
            C.c_int, C.POINTER(C.c_int), C.c_double, C.c_double, C.c_double,
            C.POINTER(C.c_longlong), C.c_longlong, C.c_longlong, C.c_longlong, C.c_int,
            C.c_int, C.POINTER(C.c_double)]
        lib.cso_trial_metrics.restype = C.c_int
        lib.cso_trial_profile.argtypes = [
            C.POINTER(C.c_float), C.c_longlong, C.c_longlong, C.c_int, C.c_int, C.c_double,
            C.c_double, C.POINTER(C.c_longlong), C.c_longlong, C.c_longlong, C.c_longlong,
            C.POINTER(C.c_double)]
        lib.cso_trial_profile.restype = C.c_int
        _ORA = lib
    return _ORA


def ref_spectrum(x: np.ndarray, dt: float) -> np.ndarray:
    """The reference's in-memory realfft + rednoise (src/datpipe.c:417-448)."""
    lib = ref_lib()
    x = np.ascontiguousarray(x, dtype=np.float32)
    pipe = lib.datpipe_create(6, 100, 6.0)
    ft = nt.FFTFile()
    rc = lib.datpipe_redfft_mem(pipe, x.ctypes.data_as(C.POINTER(C.c_float)), x.size, dt,
                                b"mem", C.byref(ft))
    if rc != 0:
        lib.datpipe_free(pipe)
        raise RuntimeError("datpipe_redfft_mem failed")
    amps = np.ctypeslib.as_array(ft.amps, shape=(2 * ft.namps,)).copy()
    lib.datpipe_free(pipe)
    return amps


def make_file(amps: np.ndarray, N: int, dt: float) -> nt.FFTFile:
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


def ref_search(amps: np.ndarray, N: int, dt: float, opts, precision: int = 0,
               collapse: bool = True) -> np.ndarray:
    """The reference CPU search_file (src/search.c:1247) on this spectrum."""
    lib = ref_lib()
    ft = make_file(amps, N, dt)
    p = opts.params(lib)
    p.precision = precision
    rem = int(opts.remove) if collapse else 0
    hrem = int(opts.harm_remove) if collapse else 0
    cl = lib.search_file(C.byref(ft), C.byref(p), opts.lofreq, opts.hifreq, opts.lobin,
                         opts.blocksize, opts.threshold, rem, opts.drtol, hrem, opts.numharm,
                         None, 0, 0, 0, None, None, 1.0, -1)
    out = nt.candidates_to_numpy(cl)
    lib.candlist_free(C.byref(cl))
    return out


def ref_chunks(amps: np.ndarray, N: int, dt: float, opts):
    """(r_lo, lodr, total, cstarts) from the reference planner."""
    lib = ref_lib()
    ft = make_file(amps, N, dt)
    p = opts.params(lib)
    r_lo, lodr, total = opts.geometry(N, dt)
    plans = nt.DirectPlanSet()
    assert lib.direct_plans_build(C.byref(plans), C.byref(p), r_lo) == 0
    cs = C.POINTER(C.c_longlong)()
    nch = C.c_longlong(0)
    assert lib.chunk_starts(C.byref(plans), C.byref(ft), C.byref(p), total, opts.blocksize,
                            C.byref(cs), C.byref(nch)) == 0
    cstarts = np.ctypeslib.as_array(cs, shape=(nch.value,)).copy()
    C.CDLL(None).free(cs)
    lib.direct_plans_free(C.byref(plans))
    return r_lo, lodr, total, cstarts


def oracle_metrics(amps: np.ndarray, N: int, dt: float, opts, t_begin: int, count: int,
                   prec64: bool = False):
    """Per-trial metrics [nslot, count] from oracle/cs_oracle.c."""
    lib = oracle_lib()
    p = opts.params(ref_lib())
    r_lo, lodr, total, cstarts = ref_chunks(amps, N, dt, opts)
    decims = np.array(list(p.decimations)[:p.ndecim], dtype=np.int32)
    nslot = 1 + int((decims > 1).sum())
    out = np.zeros((nslot, count), dtype=np.float64)
    a = np.ascontiguousarray(amps, dtype=np.float32)
    rc = lib.cso_trial_metrics(a.ctypes.data_as(C.POINTER(C.c_float)), a.size // 2, N,
                               opts.nharms, opts.m, opts.hidr, decims.size,
                               decims.ctypes.data_as(C.POINTER(C.c_int)), opts.boxcar_fsp,
                               opts.boxcar_maxfrac, r_lo,
                               cstarts.ctypes.data_as(C.POINTER(C.c_longlong)), cstarts.size,
                               total, t_begin, count, int(prec64),
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == nslot, rc
    return out, (r_lo, lodr, total, cstarts, decims)


def oracle_candidates(metrics: np.ndarray, geo, N: int, dt: float, opts, t_begin: int = 0):
    """Reference candidate emission (src/search.c:866-905, 705-716) from
    per-trial metrics: uncollapsed, in (chunk, slot, trial) order."""
    r_lo, lodr, total, cstarts, decims = geo
    T = N * dt
    nyq = N / 2.0
    ks = [1] + [int(k) for k in decims if k > 1]
    rows = []
    count = metrics.shape[1]
    t = np.arange(t_begin, t_begin + count)
    chunk = np.searchsorted(cstarts, t, side="right") - 1
    for c in np.unique(chunk):
        sel = np.nonzero(chunk == c)[0]
        i0 = int(cstarts[c])
        rstart = r_lo + float(i0) * lodr
        for s, k in enumerate(ks):
            for i in sel:
                mval = metrics[s, i]
                if not (mval > opts.threshold):
                    continue
                j = int(t[i]) - i0
                rf = rstart + float(j) * lodr
                rsel = float(k) * rf if k != 1 else rf
                if s and not (rsel < nyq):
                    continue
                rows.append((rsel / T, float(mval), rsel, opts.nharms // k, np.nan))
    return np.array(rows, dtype=nt.CAND_DTYPE)


# ---------------------------------------------------------------------------
# dedispersion: the reference's dispersion.c + the restated block driver
# ---------------------------------------------------------------------------
_DD = None


def have_dedisp_ref() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libdedisp_ref.so"))


def dedisp_ref_lib() -> C.CDLL:
    global _DD
    if _DD is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libdedisp_ref.so"))
        IP = C.POINTER(C.c_int)
        lib.odd_tables.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_int, IP, IP, IP,
                                   C.POINTER(C.c_double)]
        lib.odd_run.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, IP, IP, C.c_longlong, C.c_void_p, C.c_longlong,
                                C.POINTER(C.c_longlong)]
        _DD = lib
    return _DD


def ref_dedisp_tables(nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, L=2400):
    lib = dedisp_ref_lib()
    idisp = np.zeros(nchan, np.int32)
    offs = np.zeros((ndm, nsub), np.int32)
    bpr = C.c_int(0)
    avg = C.c_double(0)
    IP = C.POINTER(C.c_int)
    lib.odd_tables(nchan, nsub, ndm, lodm, dmstep, lofreq, chanwid, dt, 1, L,
                   idisp.ctypes.data_as(IP), offs.ctypes.data_as(IP), C.byref(bpr), C.byref(avg))
    return idisp, offs, bpr.value, avg.value


def _fresh_dedisp_lib() -> C.CDLL:
    """A private copy of libdedisp_ref.so: clip_times keeps its running
    averages in static variables (clipping.c:55-59), so every clipped run
    starts from a new instance, as a prepsubband process does."""
    import shutil
    import tempfile
    d = tempfile.mkdtemp(prefix="ddref")
    path = os.path.join(d, "libdedisp_ref.so")
    shutil.copy(os.path.join(REF_DIR, "libdedisp_ref.so"), path)
    lib = C.CDLL(path)
    IP = C.POINTER(C.c_int)
    lib.odd_run_clip.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, IP, IP, C.c_longlong, C.c_void_p, C.c_longlong,
                                 C.POINTER(C.c_longlong), C.c_float, C.POINTER(C.c_longlong)]
    lib.odd_clip_levels_to.argtypes = [C.c_void_p, C.c_longlong]
    return lib


def ref_dedisp_run(raw, nsub, idisp, offs, L, bpr, numout=-1, clip_sigma=0.0,
                   return_clipped=False, return_levels=False):
    """The reference's prepsubband output for every DM: [ndm][nout] float32.
    With clip_sigma > 0, PRESTO's clip_times runs on each raw block as
    prepsubband's -clip does; return_clipped adds the number of spectra it
    replaced, return_levels the channel levels it leaves after each block
    ([nblocks][nchan] float32, ascending frequency; rows of blocks it never
    read stay NaN)."""
    lib = dedisp_ref_lib() if clip_sigma <= 0 else _fresh_dedisp_lib()
    raw = np.ascontiguousarray(raw, np.uint8)
    nspec, nchan = raw.shape
    ndm = offs.shape[0]
    cap = nspec if numout < 0 else min(numout, nspec)
    out = np.zeros((ndm, max(cap, 1)), np.float32)
    got = C.c_longlong(0)
    nclip = C.c_longlong(0)
    IP = C.POINTER(C.c_int)
    idisp = np.ascontiguousarray(idisp, np.int32)
    offs = np.ascontiguousarray(offs, np.int32)
    levels = np.full((max(nspec // L, 1), nchan), np.nan, np.float32)
    if clip_sigma > 0:
        if return_levels:
            lib.odd_clip_levels_to(C.c_void_p(levels.ctypes.data), C.c_longlong(nspec // L))
        lib.odd_run_clip(raw.ctypes.data, nspec, nchan, nsub, ndm, L, bpr,
                         idisp.ctypes.data_as(IP), offs.ctypes.data_as(IP), cap, out.ctypes.data,
                         out.shape[1], C.byref(got), float(clip_sigma), C.byref(nclip))
        lib.odd_clip_levels_to(None, C.c_longlong(0))
    else:
        lib.odd_run(raw.ctypes.data, nspec, nchan, nsub, ndm, L, bpr, idisp.ctypes.data_as(IP),
                    offs.ctypes.data_as(IP), cap, out.ctypes.data, out.shape[1], C.byref(got))
    res = out[:, :got.value]
    extra = ((nclip.value,) if return_clipped else ()) + ((levels,) if return_levels else ())
    return (res,) + extra if extra else res
