"""ctypes bindings of the native libraries (include/coherent_search.h,
include/cs_b200.h).

The structures mirror the C layouts field for field; they are the
reference's types (CoherentSearch_C include/coherent_search.h:48-195), so the
same definitions also bind the reference library in the oracle tests.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# the built libraries; CS_B200_LIBDIR points at another build of them
LIBDIR = os.environ.get("CS_B200_LIBDIR") or os.path.join(PKG, "lib")


class SimpleInf(C.Structure):
    _fields_ = [("path", C.c_char_p), ("object", C.c_char_p), ("has_epoch", C.c_int),
                ("epoch", C.c_double), ("N", C.c_longlong), ("has_N", C.c_int),
                ("dt", C.c_double), ("has_dt", C.c_int), ("DM", C.c_double),
                ("has_DM", C.c_int)]


class FFTFile(C.Structure):
    _fields_ = [("path", C.c_char_p), ("inf", SimpleInf), ("N", C.c_longlong),
                ("T", C.c_double), ("df", C.c_double), ("dereddened", C.c_int),
                ("detrended", C.c_int), ("DC", C.c_float), ("Nyquist", C.c_float),
                ("amps", C.POINTER(C.c_float)), ("namps", C.c_longlong),
                ("map", C.c_void_p), ("mapsize", C.c_size_t), ("owns_amps", C.c_int)]


class SearchParams(C.Structure):
    _fields_ = [("nharms", C.c_int), ("m", C.c_int), ("numbetween", C.c_int),
                ("hidr", C.c_double), ("threshold", C.c_double),
                ("boxcar_fsp", C.c_double), ("boxcar_maxfrac", C.c_double),
                ("boxcar_gatemargin", C.c_double), ("ndecim", C.c_int),
                ("decimations", C.c_int * 64), ("precision", C.c_int),
                ("sigma", C.c_int)]


class Candidate(C.Structure):
    _fields_ = [("freq", C.c_double), ("metric", C.c_double), ("r", C.c_double),
                ("nharm", C.c_int), ("ducy", C.c_double)]


class CandidateList(C.Structure):
    _fields_ = [("v", C.POINTER(Candidate)), ("n", C.c_size_t), ("cap", C.c_size_t)]


class DirectPlan(C.Structure):
    _fields_ = [("h", C.c_int), ("m", C.c_int), ("q", C.c_int), ("s", C.c_int),
                ("base_adv", C.c_int), ("pnum", C.c_int), ("rfloor0", C.c_int),
                ("dr0", C.c_double), ("P", C.c_int), ("row", C.POINTER(C.c_int32)),
                ("W", C.POINTER(C.c_float)), ("A_re", C.POINTER(C.c_float)),
                ("A_im", C.POINTER(C.c_float)), ("carry", C.POINTER(C.c_uint8)),
                ("ngrp", C.c_int), ("grow", C.POINTER(C.c_int32)),
                ("goff", C.POINTER(C.c_int32)), ("gnj", C.POINTER(C.c_int32)),
                ("gW", C.POINTER(C.c_float)), ("gA_re", C.POINTER(C.c_float)),
                ("gA_im", C.POINTER(C.c_float))]


class DirectPlanSet(C.Structure):
    _fields_ = [("plans", C.POINTER(DirectPlan)), ("n", C.c_int)]


class CsB200Info(C.Structure):
    _fields_ = [("ntiles", C.c_int), ("nchunks", C.c_longlong), ("nslot", C.c_int),
                ("npad", C.c_int), ("kpad", C.c_int), ("smem_bytes", C.c_int),
                ("grid", C.c_int), ("total", C.c_longlong), ("rec_capacity", C.c_uint),
                ("kernel", C.c_int)]


CAND_DTYPE = np.dtype([("freq", "f8"), ("metric", "f8"), ("r", "f8"), ("nharm", "i4"),
                       ("ducy", "f8")], align=True)
assert CAND_DTYPE.itemsize == C.sizeof(Candidate)


def declare_host_api(lib: C.CDLL) -> C.CDLL:
    """Prototypes of the coherent_search.h host API (ours or the reference's)."""
    P = C.POINTER
    lib.params_defaults.argtypes = [P(SearchParams)]
    if hasattr(lib, "cs_prep_pad_value"):
        lib.cs_prep_pad_value.argtypes = [P(C.c_float), C.c_longlong]
        lib.cs_prep_pad_value.restype = C.c_double
    lib.decimation_set.argtypes = [C.c_int, C.c_int, P(C.c_int), C.c_int]
    lib.decimation_set.restype = C.c_int
    lib.trial_grid_rational.argtypes = [C.c_double, P(C.c_int), P(C.c_int)]
    lib.trial_grid_rational.restype = C.c_int
    lib.direct_plans_build.argtypes = [P(DirectPlanSet), P(SearchParams), C.c_double]
    lib.direct_plans_build.restype = C.c_int
    lib.direct_plans_free.argtypes = [P(DirectPlanSet)]
    lib.chunk_starts.argtypes = [P(DirectPlanSet), P(FFTFile), P(SearchParams), C.c_longlong,
                                 C.c_int, P(P(C.c_longlong)), P(C.c_longlong)]
    lib.chunk_starts.restype = C.c_int
    lib.cs_harmonic_fits.argtypes = [P(DirectPlan), P(FFTFile), P(SearchParams), C.c_longlong]
    lib.cs_harmonic_fits.restype = C.c_int
    lib.ladder_boxcar_widths.argtypes = [C.c_int, C.c_int, P(SearchParams), P(C.c_int), C.c_int]
    lib.ladder_boxcar_widths.restype = C.c_int
    lib.analytic_sigma.argtypes = [P(C.c_uint8), C.c_int, C.c_int]
    lib.analytic_sigma.restype = C.c_double
    lib.boxcar_shape.argtypes = [P(C.c_double), C.c_int, P(C.c_int), C.c_int, P(C.c_uint8),
                                 C.c_int, C.c_int]
    lib.candlist_free.argtypes = [P(CandidateList)]
    lib.remove_duplicates.argtypes = [P(CandidateList), C.c_double]
    lib.remove_duplicates.restype = CandidateList
    lib.remove_harmonics.argtypes = [P(CandidateList), C.c_int, C.c_double]
    lib.remove_harmonics.restype = CandidateList
    lib.write_candidates.argtypes = [P(CandidateList), C.c_char_p, C.c_double]
    lib.write_candidates.restype = C.c_int
    lib.measure_ducy.argtypes = [P(FFTFile), P(CandidateList), P(SearchParams)]
    lib.measure_ducy.restype = CandidateList
    lib.search_file.argtypes = [P(FFTFile), P(SearchParams), C.c_double, C.c_double, C.c_int,
                                C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int,
                                C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_void_p,
                                C.c_double, C.c_int]
    lib.search_file.restype = CandidateList
    return lib


def declare_gpu_api(lib: C.CDLL) -> C.CDLL:
    """Prototypes of libcsgpu.so (the reference GPU ABI plus cs_b200.h)."""
    P = C.POINTER
    lib.cs_gpu_available.argtypes = [C.c_int, C.c_char_p, C.c_size_t]
    lib.cs_gpu_available.restype = C.c_int
    lib.cs_gpu_session_create.argtypes = [P(FFTFile), P(SearchParams), P(DirectPlanSet),
                                          P(C.c_longlong), C.c_longlong, C.c_int, C.c_longlong,
                                          C.c_double, C.c_double, C.c_int]
    lib.cs_gpu_session_create.restype = C.c_void_p
    lib.cs_gpu_session_matches.argtypes = [C.c_void_p, P(FFTFile), P(SearchParams), C.c_int,
                                           C.c_longlong, C.c_double, C.c_double, C.c_int]
    lib.cs_gpu_session_matches.restype = C.c_int
    lib.cs_gpu_session_run.argtypes = [C.c_void_p, P(FFTFile), C.c_double]
    lib.cs_gpu_session_run.restype = CandidateList
    lib.cs_gpu_session_free.argtypes = [C.c_void_p]
    lib.cs_gpu_search_region.argtypes = [P(FFTFile), P(SearchParams), P(DirectPlanSet),
                                         P(C.c_longlong), C.c_longlong, C.c_int, C.c_longlong,
                                         C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.cs_gpu_search_region.restype = CandidateList
    lib.cs_b200_session_info.argtypes = [C.c_void_p, P(CsB200Info)]
    lib.cs_b200_session_info.restype = C.c_int
    lib.cs_b200_session_device_amps.argtypes = [C.c_void_p]
    lib.cs_b200_session_device_amps.restype = C.c_void_p
    lib.cs_b200_multi_enqueue.argtypes = [C.POINTER(C.c_void_p), C.c_int,
                                          C.POINTER(C.c_void_p), C.c_double, C.c_void_p]
    lib.cs_b200_multi_enqueue.restype = C.c_int
    lib.cs_b200_multi_graph_create.argtypes = [C.POINTER(C.c_void_p), C.c_int,
                                               C.POINTER(C.c_void_p), C.c_double]
    lib.cs_b200_multi_graph_create.restype = C.c_void_p
    lib.cs_b200_multi_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    lib.cs_b200_multi_graph_launch.restype = C.c_int
    lib.cs_b200_multi_graph_free.argtypes = [C.c_void_p]
    lib.cs_b200_multi_graph_free.restype = None
    lib.cs_b200_session_enqueue_device.argtypes = [C.c_void_p, C.c_void_p, C.c_double,
                                                   C.c_void_p]
    lib.cs_b200_session_enqueue_device.restype = C.c_int
    lib.cs_b200_session_collect.argtypes = [C.c_void_p, C.c_double, P(CandidateList),
                                            P(C.c_float)]
    lib.cs_b200_session_collect.restype = C.c_int
    lib.cs_b200_session_collect_collapsed.argtypes = [C.c_void_p, C.c_double, C.c_int,
                                                      C.c_double, C.c_int, C.c_int, C.c_double,
                                                      P(CandidateList), P(C.c_float)]
    lib.cs_b200_session_collect_collapsed.restype = C.c_int
    lib.cs_b200_session_collapse_enqueue.argtypes = [C.c_void_p, C.c_double, C.c_int,
                                                     C.c_double, C.c_int, C.c_int, C.c_double]
    lib.cs_b200_session_collapse_enqueue.restype = C.c_int
    lib.cs_b200_session_collapse_wait.argtypes = [C.c_void_p, P(CandidateList), P(C.c_float)]
    lib.cs_b200_session_collapse_wait.restype = C.c_int
    lib.cs_b200_session_sync.argtypes = [C.c_void_p]
    lib.cs_b200_session_sync.restype = C.c_int
    lib.cs_b200_session_park_drain.argtypes = []
    lib.cs_b200_session_park_drain.restype = C.c_int
    lib.cs_b200_session_search_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_double,
                                                   C.c_void_p, C.c_longlong,
                                                   P(C.c_longlong), C.c_void_p]
    lib.cs_b200_session_search_noalloc.restype = C.c_int
    lib.cs_gpu_batch_create.argtypes = [C.c_int, C.c_int, C.c_size_t]
    lib.cs_gpu_batch_create.restype = C.c_void_p
    lib.cs_gpu_batch_submit.argtypes = [C.c_void_p, P(FFTFile), P(SearchParams), C.c_double,
                                        C.c_double, C.c_int, C.c_int, C.c_double]
    lib.cs_gpu_batch_submit.restype = C.c_longlong
    lib.cs_gpu_batch_wait.argtypes = [C.c_void_p, C.c_longlong, P(CandidateList),
                                      P(C.c_double), P(C.c_double)]
    lib.cs_gpu_batch_wait.restype = C.c_int
    lib.cs_gpu_batch_warm.argtypes = [C.c_void_p, P(FFTFile), P(SearchParams), C.c_double,
                                      C.c_double, C.c_int, C.c_int]
    lib.cs_gpu_batch_warm.restype = C.c_int
    lib.cs_gpu_batch_device_bytes.argtypes = [C.c_void_p]
    lib.cs_gpu_batch_device_bytes.restype = C.c_longlong
    lib.cs_gpu_batch_cancel.argtypes = [C.c_void_p, C.c_longlong]
    lib.cs_gpu_batch_cancel.restype = C.c_int
    lib.cs_gpu_batch_pending.argtypes = [C.c_void_p]
    lib.cs_gpu_batch_pending.restype = C.c_int
    lib.cs_gpu_batch_free.argtypes = [C.c_void_p]
    lib.cs_spectrum_create.argtypes = [C.c_longlong, C.c_double, C.c_int, C.c_int, C.c_double,
                                       C.c_int]
    lib.cs_spectrum_create.restype = C.c_void_p
    lib.cs_spectrum_run_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cs_spectrum_run_device.restype = C.c_int
    lib.cs_spectrum_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cs_spectrum_run.restype = C.c_int
    lib.cs_spectrum_free.argtypes = [C.c_void_p]
    lib.cs_ducy_create.argtypes = [C.c_double, C.c_double, C.c_int]
    lib.cs_ducy_create.restype = C.c_void_p
    lib.cs_ducy_run_device.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong,
                                       C.c_void_p, C.c_longlong, P(C.c_double), C.c_void_p]
    lib.cs_ducy_run_device.restype = C.c_int
    lib.cs_ducy_free.argtypes = [C.c_void_p]
    lib.cs_clip_scratch_bytes.argtypes = [C.c_longlong, C.c_int]
    lib.cs_clip_scratch_bytes.restype = C.c_size_t
    lib.cs_clip_count.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_float,
                                  P(C.c_longlong), C.c_void_p, C.c_void_p, C.c_size_t,
                                  C.c_void_p, C.c_int]
    lib.cs_clip_count.restype = C.c_int
    lib.cs_clip_levels.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_float,
                                   P(C.c_longlong), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_size_t, C.c_void_p, C.c_int]
    lib.cs_clip_levels.restype = C.c_int
    IP = P(C.c_int)
    lib.cs_dedisp_tables.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_int, IP, IP, IP,
                                     P(C.c_double)]
    lib.cs_dedisp_tables.restype = C.c_int
    lib.cs_dedisp_create.argtypes = [C.c_int, C.c_int, C.c_int, IP, IP, C.c_int, C.c_int,
                                     C.c_longlong, C.c_int]
    lib.cs_dedisp_create.restype = C.c_void_p
    lib.cs_dedisp_output_length.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong]
    lib.cs_dedisp_output_length.restype = C.c_longlong
    lib.cs_dedisp_run_device.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong,
                                         C.c_void_p, C.c_longlong, C.c_void_p,
                                         P(C.c_longlong)]
    lib.cs_dedisp_run_device.restype = C.c_int
    lib.cs_dedisp_run_device_clipped.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong,
                                                 C.c_longlong, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_longlong, C.c_void_p,
                                                 P(C.c_longlong)]
    lib.cs_dedisp_run_device_clipped.restype = C.c_int
    lib.cs_dedisp_run.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong,
                                  C.c_void_p, C.c_longlong, P(C.c_longlong)]
    lib.cs_dedisp_run.restype = C.c_int
    lib.cs_dedisp_last_times.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float)]
    lib.cs_dedisp_last_times.restype = C.c_int
    lib.cs_dedisp_free.argtypes = [C.c_void_p]
    return lib


_GPU = None
_HOST = None


def gpu_lib() -> C.CDLL:
    """libcsgpu.so; raises if the extension has not been built."""
    global _GPU
    if _GPU is None:
        path = os.path.join(LIBDIR, "libcsgpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `python -m coherentsearch_c_b200.build`")
        _GPU = declare_gpu_api(C.CDLL(path))
    return _GPU


def host_lib() -> C.CDLL:
    global _HOST
    if _HOST is None:
        gpu_lib()
        path = os.path.join(LIBDIR, "libcoherent_search.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `python -m coherentsearch_c_b200.build`")
        _HOST = declare_host_api(C.CDLL(path))
    return _HOST


def candidates_to_numpy(cl: CandidateList) -> np.ndarray:
    n = int(cl.n)
    if n == 0:
        return np.zeros(0, dtype=CAND_DTYPE)
    raw = (C.c_char * (n * C.sizeof(Candidate))).from_address(C.cast(cl.v, C.c_void_p).value)
    return np.frombuffer(raw, dtype=CAND_DTYPE).copy()
