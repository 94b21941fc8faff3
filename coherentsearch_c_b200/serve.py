"""Search request loop over the batched engine (cs_gpu_batch_*).

Requests of any length and harmonic count arrive while others run. The
server admits each one to a batch slot as soon as a slot, and device memory
within the budget, is free. Searches in different slots overlap on the GPU:
one slot's table building and upload run beside another's kernel. Each
request returns a future that resolves to its raw candidates and its latency
(arrival to result).

    with SearchServer(nslots=3) as srv:
        fut = srv.submit(amps, N, dt, Options(nharms=32))
        cands, latency_ms = fut.result()

`PlainServer` serves the same requests one at a time, with a session created
and freed per request (the reference's single-file GPU form). It is the
baseline that `run_stream` reports beside the server.
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import threading
import time
from dataclasses import dataclass

import numpy as np

from .batch import Batch
from .search import Options, Session


@dataclass
class Request:
    amps: np.ndarray          # interleaved float32 spectrum (kept alive by the caller)
    N: int
    dt: float
    opts: Options

    @property
    def trials(self) -> int:
        return int(self.opts.geometry(self.N, self.dt)[2])


class SearchServer:
    """Continuous batching on one GPU: a Batch plus waiter threads that turn
    completions into futures as they happen (not in submission order)."""

    def __init__(self, nslots: int = 3, mem_budget: int = 0, device: int = 0):
        self.batch = Batch(device=device, nslots=nslots, mem_budget=mem_budget)
        # one waiter per in-flight request, so a result is seen when it lands
        self.pool = cf.ThreadPoolExecutor(max_workers=64)
        self.lock = threading.Lock()
        self.stats: list[tuple[float, float]] = []   # (ms queued for a slot, ms on the slot)

    def submit(self, amps, N: int, dt: float, opts: Options | None = None,
               arrival: float | None = None) -> cf.Future:
        t0 = time.perf_counter() if arrival is None else arrival
        with self.lock:
            rid = self.batch.submit(amps, N, dt, opts)

        def finish():
            cands, queued, run = self.batch.wait(rid)
            with self.lock:
                self.stats.append((queued, run))
            return cands, 1e3 * (time.perf_counter() - t0)

        return self.pool.submit(finish)

    def warm(self, N: int, dt: float, opts: Options | None = None) -> None:
        """Grow every slot's device buffers to the largest request expected
        (length N with `opts`; nharms 60 needs the largest tables) before
        traffic arrives.  A slot that grows while serving frees and allocates
        device memory, and cudaFree waits for the whole device, so the other
        slots' requests stall behind it."""
        self.batch.warm(N, dt, opts or Options())

    def close(self) -> None:
        self.pool.shutdown(wait=True)
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class PlainServer:
    """One request at a time: create a session, search, free it."""

    def __init__(self, device: int = 0):
        self.device = device
        self.pool = cf.ThreadPoolExecutor(max_workers=1)

    def submit(self, amps, N: int, dt: float, opts: Options | None = None,
               arrival: float | None = None) -> cf.Future:
        t0 = time.perf_counter() if arrival is None else arrival

        def run():
            ses = Session(N, dt, opts or Options(), device=self.device)
            try:
                cands = ses.run_raw(amps)
            finally:
                ses.close()
            return cands, 1e3 * (time.perf_counter() - t0)

        return self.pool.submit(run)

    def close(self) -> None:
        self.pool.shutdown(wait=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (s from the start) of a Poisson process of `rate` per s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def run_stream(server, requests: list[Request], arrivals: np.ndarray) -> dict:
    """Submit each request at its arrival time; return latency percentiles
    (ms, arrival to result), throughput (trials/s over first arrival to last
    result) and the results in request order."""
    start = time.perf_counter()
    futs = []
    for req, at in zip(requests, arrivals):
        delay = start + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        futs.append(server.submit(req.amps, req.N, req.dt, req.opts, arrival=start + at))
    results = [f.result() for f in futs]
    end = time.perf_counter()
    lat = np.array([r[1] for r in results])
    trials = sum(r.trials for r in requests)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "requests": len(requests),
            "trials": trials, "wall_s": end - start, "trials_per_s": trials / (end - start),
            "results": [r[0] for r in results]}


def log_uniform_lengths(n: int, lo: int, hi: int, seed: int, quantum: int = 1024) -> list[int]:
    rng = np.random.default_rng(seed)
    return [max(quantum, int(math.exp(rng.uniform(math.log(lo), math.log(hi)))) // quantum * quantum)
            for _ in range(n)]
