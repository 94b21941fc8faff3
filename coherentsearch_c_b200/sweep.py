"""A list of spectra searched in groups, one persistent launch per group.

This is the device form of the reference's list driver (src/cli.c:976-1099,
src/search.c:1292-1341), which searches one file per call.  Here the
spectra of a group go through one launch of the warp-specialised kernel
over a single list of (spectrum, tile) work items (cs_b200_multi_enqueue);
while a group runs, the host builds the next group's tables, so table
builds, uploads and candidate harvests overlap the kernels.  Sessions are
reused through the library's session park (CS_B200_SESSION_PARK must allow
two groups).

`autotune` picks the group size from measured times on a sample of the
list and remembers it per geometry class (harmonic count, length range).
"""
from __future__ import annotations

import json
import os
import time

from .search import Options, Session, multi_collect, multi_enqueue


def search_list(spectra, dt: float, opts: Options, group: int, device: int = 0,
                upload=None, stream=None):
    """Search every spectrum of `spectra`, a list of (N, device pointer) with
    namps = N/2 float2 at each pointer, in groups of `group`.  `upload(i)`,
    if given, returns spectrum i's device pointer instead (it is called one
    group ahead, so its copies overlap the previous group's kernel; queue
    them on `stream`, the cudaStream_t handle the launches follow).  Returns
    the raw candidate arrays in list order."""
    n = len(spectra)
    outs = [None] * n

    def harvest(done):
        pidx, psess, pptrs = done
        res, _ = multi_collect(psess, pptrs)
        for i, r in zip(pidx, res):
            outs[i] = r
        for s in psess:
            s.close()

    prev = None
    for g0 in range(0, n, max(1, group)):
        idx = list(range(g0, min(n, g0 + group)))
        # host tables of this group while the previous group's kernel runs
        sess = [Session(spectra[i][0], dt, opts, device=device) for i in idx]
        ptrs = [upload(i) if upload else spectra[i][1] for i in idx]
        # queued behind the previous launch; its harvest then overlaps this one
        multi_enqueue(sess, ptrs, stream=stream)
        if prev is not None:
            harvest(prev)
        prev = (idx, sess, ptrs)
    if prev is not None:
        harvest(prev)
    return outs


def warm(max_n: int, dt: float, opts: Options, count: int, device: int = 0) -> None:
    """Park `count` sessions sized for the longest spectrum of a list, so that
    the groups of search_list reload them without growing a device buffer
    (a cudaFree waits for the whole device).  The park must hold `count`
    (CS_B200_SESSION_PARK); cs_b200_session_park_drain gives the memory back."""
    sess = [Session(max_n, dt, opts, device=device) for _ in range(count)]
    for s in sess:
        s.close()


def geometry_class(lengths, nharms: int) -> str:
    lo, hi = min(lengths), max(lengths)
    return f"nh{nharms}_N{lo.bit_length() - 1}-{hi.bit_length() - 1}"


def autotune(spectra, dt: float, opts: Options, candidates=(1, 2, 4, 8, 16, 32),
             sample: int = 16, cache_path: str | None = None, device: int = 0,
             upload=None, stream=None, sync=None):
    """Time search_list on the first `sample` spectra for each group size and
    return (best group size, {group: seconds}).  With `cache_path` the choice
    is stored per geometry class and reused.  `sync()` waits for the device
    (e.g. torch.cuda.synchronize) before each clock reading."""
    key = geometry_class([N for N, _ in spectra], opts.nharms)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            return int(cache[key]["group"]), cache[key]["times"]
    sub = spectra[:sample]
    times = {}
    search_list(sub, dt, opts, max(candidates), device, upload, stream)    # warm
    for g in candidates:
        if g > len(sub):
            continue
        best_t = None
        for _ in range(2):                  # best of two: the host side is noisy
            if sync:
                sync()
            t0 = time.perf_counter()
            search_list(sub, dt, opts, g, device, upload, stream)
            if sync:
                sync()
            dtm = time.perf_counter() - t0
            best_t = dtm if best_t is None else min(best_t, dtm)
        times[g] = best_t
    best = min(times, key=times.get)
    if cache_path:
        cache[key] = {"group": best, "times": {str(k): v for k, v in times.items()}}
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1)
    return best, times
