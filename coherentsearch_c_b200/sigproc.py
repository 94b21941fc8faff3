"""SIGPROC filterbank files for the raw-data front end.

read_header parses the header with cs_sigproc_read_header (libcoherent_search.so,
restating PRESTO's read_filterbank_header, third_party/presto/src/sigproc_fb.c:240-345)
and open_filterbank maps the 8-bit payload as [nspectra][nchans], highest
frequency first, the layout the dedispersion takes.  dedisp_tables_for builds
the prepsubband delay tables from the header's band (PRESTO's lo_freq and
|foff|, :435-441) and sample time.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as nt


class CsSigproc(C.Structure):
    _fields_ = [("nchans", C.c_int), ("nbits", C.c_int), ("nifs", C.c_int), ("ibeam", C.c_int),
                ("telescope_id", C.c_int), ("machine_id", C.c_int), ("signedints", C.c_int),
                ("tstart", C.c_double), ("tsamp", C.c_double), ("fch1", C.c_double),
                ("foff", C.c_double), ("src_raj", C.c_double), ("src_dej", C.c_double),
                ("source_name", C.c_char * 80), ("rawdatafile", C.c_char * 80),
                ("header_bytes", C.c_longlong), ("nspectra", C.c_longlong),
                ("lofreq", C.c_double), ("chanwid", C.c_double)]


def read_header(path: str) -> dict:
    lib = nt.host_lib()
    lib.cs_sigproc_read_header.argtypes = [C.c_char_p, C.POINTER(CsSigproc)]
    lib.cs_sigproc_read_header.restype = C.c_int
    h = CsSigproc()
    if lib.cs_sigproc_read_header(str(path).encode(), C.byref(h)) != 0:
        raise ValueError(f"{path}: not a filterbank the device front end takes (see stderr)")
    out = {f: getattr(h, f) for f, _ in CsSigproc._fields_}
    out["source_name"] = h.source_name.decode(errors="replace")
    out["rawdatafile"] = h.rawdatafile.decode(errors="replace")
    return out


def open_filterbank(path: str):
    """(header, np.memmap [nspectra][nchans] uint8)."""
    h = read_header(path)
    data = np.memmap(path, dtype=np.uint8, mode="r", offset=h["header_bytes"],
                     shape=(h["nspectra"], h["nchans"]))
    return h, data


def dedisp_tables_for(header: dict, nsub: int, ndm: int, lodm: float, dmstep: float,
                      spectra_per_subint: int = 2400):
    """prepsubband's delay tables for this file (SIGPROC blocks of 2400)."""
    from .dedisp import dedisp_tables
    return dedisp_tables(header["nchans"], nsub, ndm, lodm, dmstep, header["lofreq"],
                         header["chanwid"], header["tsamp"], spectra_per_subint)
