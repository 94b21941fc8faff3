"""Benchmark: Fourier trials/s of the coherent harmonic-sum search on B200.

Workload (one step = one full search of one spectrum): a float32 time series
of N = 2^23 samples at dt = 64 us (Gaussian noise, power-law red noise of
index -2, pulsars at 1.7 / 29.4 / 311 Hz), nharms = 60, m = 16, hidr = 0.5,
lofreq 0.1 Hz .. hifreq 125 Hz (8,046,622 trials), decimations k = 1..6,
blocksize 65536, threshold 8.  Synthetic and seeded; the spectrum is a
normalised real FFT of the series (numpy) in PRESTO packing.

Arms:
  default          the B200 kernels (libcsgpu.so)
  --impl reference the reference's own OpenMP/AVX-512 CPU search path
                   (oracle/_ref, built from the reference sources), on all
                   host cores, same workload and metric

JSON line (rank 0): value = trials/s with the spectrum resident in HBM (each
step: enqueue + candidate readback + ordering), e2e = the same through
cs_gpu_session_run with the spectrum in pinned host memory (H2D + search +
D2H inside the timed region).  Steps are timed with CUDA events, L2 is
flushed (512 MiB write) before every timed step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "precision-study single file: N=2^23 f32 series, dt=64us, nharms=60, m=16, "
                "hidr=0.5, 0.1-125 Hz, maxdecim 6, threshold 8",
    "N": 1 << 23, "dt": 64e-6, "nharms": 60, "m": 16,
    "l2": "flushed (512 MiB write) before each timed step",
}
# Trials per chunk (--blocksize) of each arm.  It sets how the trials are
# batched, not which trials run or what they give: chunks also break at every
# harmonic change point, so each chunk's harmonic set, noise scale and
# candidates are the same at any blocksize.  Each arm runs its own best: the
# GPU 65536 (the reference's GPU default, src/cli.c:920), the CPU 2048 (2.5x
# faster than 65536 there, its cache-sized batches).
BLOCKSIZE_GPU = 65536
BLOCKSIZE_CPU = 2048
METRIC = "Fourier trials/sec/GPU"
UNIT = "trials/s"
DFT_FLOP_PER_TRIAL = 28560.0      # 2*(2nh-1)*2nh at nh=60 (k | nh folds add none)
SIMT_OPS_PER_TRIAL = 6000.0       # interp 1920 FMA + 360 rotate + boxcar/fold ~3700


KERNEL_NAMES = {0: "cs_search_kernel", 1: "search_ws_cfg60", 2: "search_f64",
                3: "search_tma_cfg60", 4: "interp_tc + search_pre_cfg60"}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return pk.get("hbm_gbs", 6650.0), pk.get("bf16_tflops", 1590.0), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        # the samples are summarised into the JSON line; the raw file goes to
        # CS_B200_CLOCKS_DIR when set (to keep it), else the temp directory
        import tempfile
        self.path = os.path.join(os.environ.get("CS_B200_CLOCKS_DIR") or tempfile.gettempdir(),
                                 f"cs_b200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx.append(float(r[2]))
                for i, n in enumerate(names):
                    if r[5 + i].strip() == "Active":
                        reasons.add(n)
            except Exception:
                pass
        if sm:
            loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
            out["sm_mhz"] = statistics.median(loaded)
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        return out


def make_spectrum():
    from coherentsearch_c_b200 import synth
    x = synth.make_series(synth.config_precision(N=WORKLOAD["N"]))
    return synth.amps_interleaved(synth.normalised_spectrum(x)), x.size


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def cpu_reference_rate(amps, N, seconds=10.0, max_reps=50):
    """The reference CPU search_file (OpenMP, all host threads) on the full
    workload, repeated for about `seconds`; returns (trials/s, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    from coherentsearch_c_b200.search import Options
    opts = Options(blocksize=BLOCKSIZE_CPU, threshold=8.0)
    _, _, total = opts.geometry(N, WORKLOAD["dt"])
    cores = os.cpu_count() or 1
    rb.ref_lib()
    rb.pin_ref_threads(cores)                          # speed, not parity: every host thread
    rb.ref_search(amps, N, WORKLOAD["dt"], opts)      # warm (plans, pages)
    t0 = time.perf_counter()
    reps = 0
    while reps < max_reps:
        rb.ref_search(amps, N, WORKLOAD["dt"], opts)
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    sample = (f"{reps} full searches of the workload spectrum ({total} trials each) "
              f"with the reference CPU path (blocksize {BLOCKSIZE_CPU}, its CPU default)")
    return total * reps / dt, cores, sample


def _ref_process(path, N, dt, barrier, results):
    """One process of the reference's process-per-core deployment: one
    OpenMP thread, one search of the spectrum at `path` after the barrier."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    from coherentsearch_c_b200.search import Options
    amps = np.ascontiguousarray(np.load(path))
    opts = Options(blocksize=BLOCKSIZE_CPU, threshold=8.0)
    rb.ref_lib()
    rb.pin_ref_threads(1)
    barrier.wait()
    t0 = time.perf_counter()
    rb.ref_search(amps, N, dt, opts)
    results.put(time.perf_counter() - t0)


def _ref_one_thread(path, N, dt, results):
    """The reference CPU path on one thread, in a process of its own that
    loads the build whose FFT shim counts its transforms' time: (seconds of
    the search, seconds in the FFT, FFT calls)."""
    import ctypes as C
    os.environ["CS_REF_LIBNAME"] = "libcsref_timed.so"
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    from coherentsearch_c_b200.search import Options
    amps = np.ascontiguousarray(np.load(path))
    opts = Options(blocksize=BLOCKSIZE_CPU, threshold=8.0)
    lib = rb.ref_lib()
    lib.cs_shim_fft_seconds.argtypes = [C.POINTER(C.c_longlong), C.c_int]
    lib.cs_shim_fft_seconds.restype = C.c_double
    rb.pin_ref_threads(1)
    calls = C.c_longlong(0)
    lib.cs_shim_fft_seconds(C.byref(calls), 1)
    t0 = time.perf_counter()
    rb.ref_search(amps, N, dt, opts)
    wall = time.perf_counter() - t0
    fft = lib.cs_shim_fft_seconds(C.byref(calls), 1)
    results.put((wall, fft, int(calls.value)))


def _collect(queue, procs, n, timeout=600.0):
    """n results from worker processes; an error if they all end (or the
    time runs out) first.  The workers are joined, and ended if still
    running, in every case."""
    import queue as queue_mod
    out = []
    try:
        deadline = time.perf_counter() + timeout
        while len(out) < n:
            try:
                out.append(queue.get(timeout=1.0))
            except queue_mod.Empty:
                if time.perf_counter() > deadline or not any(p.is_alive() for p in procs):
                    raise RuntimeError(f"{n - len(out)} reference processes ended "
                                       "without a result")
    finally:
        for p in procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()
    return out


def cpu_reference_forms(amps, N, nproc=None):
    """The reference CPU path in its other two forms: one thread, and one
    single-threaded process per host core each searching the whole spectrum
    (the process-per-core deployment its README describes).  Processes are
    spawned, never forked, so a CUDA context in this process is not copied.
    Returns {"one_thread": ..., "processes": ...} in trials/s."""
    import multiprocessing as mp
    import tempfile
    from coherentsearch_c_b200.search import Options
    dt = WORKLOAD["dt"]
    opts = Options(blocksize=BLOCKSIZE_CPU, threshold=8.0)
    _, _, total = opts.geometry(N, dt)
    nproc = nproc or (os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "amps.npy")
        np.save(path, np.ascontiguousarray(amps))
        q1 = ctx.Queue()
        p1 = ctx.Process(target=_ref_one_thread, args=(path, N, dt, q1))
        p1.start()
        wall1, fft1, calls1 = _collect(q1, [p1], 1)[0]
        one = total / wall1
        barrier = ctx.Barrier(nproc)
        results = ctx.Queue()
        procs = [ctx.Process(target=_ref_process, args=(path, N, dt, barrier, results))
                 for _ in range(nproc)]
        for p in procs:
            p.start()
        times = _collect(results, procs, nproc)
    return {"one_thread": {"value": one, "cores": 1,
                           "sample": f"one full search ({total} trials), one OpenMP thread",
                           # the FFT shim's share of the search, against the
                           # reference README's single-thread split with FFTW
                           # (base + decimated c2r 0.57 of 1.33 s)
                           "fft_seconds": fft1, "fft_calls": calls1,
                           "fft_share": fft1 / wall1, "fft_share_readme_fftw": 0.57 / 1.33},
            "processes": {"value": nproc * total / max(times), "cores": nproc,
                          "sample": f"{nproc} single-threaded processes, each one full search "
                                    f"({total} trials), started together; slowest "
                                    f"{max(times):.2f} s"}}


def precision_study(ses, amps, N, dt, opts, device):
    """The FP32 search (tensor-core fp16-split DFT) against this repository's
    FP64 search (--precision f64: FP64 DFT, folds and boxcar), the FP64
    oracle, on the workload spectrum: relative S/N error of every raw
    candidate both report, the ones only one reports (threshold flips), and
    the collapsed list side by side."""
    from dataclasses import replace
    from coherentsearch_c_b200.search import Session
    raw32 = ses.run_raw(amps)
    s64 = Session(N, dt, replace(opts, precision=1), device=device)
    try:
        raw64 = s64.run_raw(amps)
        s64.enqueue(s64.device_amps_ptr())
        _, f64_ms, _ = s64.collect()
        col64 = s64.collapse(raw64)
    finally:
        s64.close()
    col32 = ses.collapse(raw32)

    def keyed(c):
        return {(round(float(r), 9), int(h)): float(m)
                for r, h, m in zip(c["r"], c["nharm"], c["metric"])}
    k32, k64 = keyed(raw32), keyed(raw64)
    common = sorted(set(k32) & set(k64))
    rel = np.array([abs(k32[k] - k64[k]) / abs(k64[k]) for k in common]) if common else np.zeros(1)
    flips = [k32.get(k, k64.get(k)) for k in set(k32) ^ set(k64)]
    thr = opts.threshold
    c64 = keyed(col64)
    table = []
    for c in col32:
        k = (round(float(c["r"]), 9), int(c["nharm"]))
        m64 = c64.get(k)
        table.append({"freq_hz": round(float(c["freq"]), 9), "nharm": int(c["nharm"]),
                      "snr_f32": round(float(c["metric"]), 6),
                      "snr_f64": None if m64 is None else round(m64, 6),
                      "rel_err": None if m64 is None else abs(float(c["metric"]) - m64) / abs(m64)})
    return {"oracle": "this repository's --precision f64 search on the GPU",
            "raw_candidates_f32": int(raw32.size), "raw_candidates_f64": int(raw64.size),
            "max_rel_snr_err": float(rel.max()), "median_rel_snr_err": float(np.median(rel)),
            "threshold_flips": len(flips),
            "flips_outside_1e-3_band": sum(1 for m in flips if abs(m - thr) > 1e-3 * thr),
            "f64_kernel_ms": f64_ms, "collapsed": table}


def ducy_timing(ses, cands, amps, N, dt, reps=3):
    """Duty cycles (measure_ducy) of the step's raw candidates: on the GPU
    from the session's resident spectrum, and by the reference's own host
    code (oracle/_ref/libcsref.so) on the same list; equal widths checked."""
    import ctypes as C
    from coherentsearch_c_b200 import native as nt
    from coherentsearch_c_b200.search import Options
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    ses.measure_ducy(cands[:8])                       # plan + tables
    t0 = time.perf_counter()
    for _ in range(reps):
        got = ses.measure_ducy(cands)["ducy"]
    gpu_ms = 1e3 * (time.perf_counter() - t0) / reps
    lib = rb.ref_lib()
    ft = rb.make_file(amps, N, dt)
    p = Options().params(lib)
    buf = (nt.Candidate * max(cands.size, 1))()
    C.memmove(buf, cands.ctypes.data, cands.size * C.sizeof(nt.Candidate))
    cl = nt.CandidateList(C.cast(buf, C.POINTER(nt.Candidate)), cands.size, cands.size)
    t0 = time.perf_counter()
    res = lib.measure_ducy(C.byref(ft), C.byref(cl), C.byref(p))
    host_ms = 1e3 * (time.perf_counter() - t0)
    ref = nt.candidates_to_numpy(res)["ducy"]
    lib.candlist_free(C.byref(res))
    return {"candidates": int(cands.size), "gpu_ms": gpu_ms, "reference_host_ms": host_ms,
            "equal": bool(np.array_equal(got, ref, equal_nan=True)),
            "note": "GPU: cs_ducy_run_device on the session's resident spectrum, host wall "
                    "time with the candidate upload and result readback; reference: its "
                    "measure_ducy on one host thread"}


def reference_gpu_rate(amps, N, dt, opts, ours=None, reps=3):
    """The reference's own GPU form (src/cuda.cu built for sm_100a,
    oracle/_ref/libcsref_gpu.so) through its search_file on the same
    spectrum: a session per call (the plain single-file form) and a session
    kept in its SearchCache (equal-length files).  Host wall time per call,
    spectrum upload included, like `e2e`."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    if not rb.have_ref_gpu():
        return {"unavailable": "oracle/_ref/libcsref_gpu.so not built"}
    _, _, total = opts.geometry(N, dt)
    rb.ref_search_gpu(amps, N, dt, opts)           # warm: context, cuFFT, pages
    t0 = time.perf_counter()
    for _ in range(reps):
        per_call = rb.ref_search_gpu(amps, N, dt, opts)
    per_s = (time.perf_counter() - t0) / reps
    srch = rb.RefGpuSearcher(opts)
    try:
        srch.search(amps, N, dt)
        t0 = time.perf_counter()
        for _ in range(reps):
            cached = srch.search(amps, N, dt)
        cached_s = (time.perf_counter() - t0) / reps
    finally:
        srch.close()
    out = {"per_file_trials_per_s": total / per_s, "cached_trials_per_s": total / cached_s,
           "per_file_ms": 1e3 * per_s, "cached_ms": 1e3 * cached_s,
           "candidates": int(cached.size),
           "source": "reference src/cuda.cu (cuFFT c2r) built for sm_100a, called through "
                     "its search_file with collapse; host wall time per call"}
    if ours is not None:
        ka = set(zip(np.round(ours["r"], 9), ours["nharm"]))
        kb = set(zip(np.round(cached["r"], 9), cached["nharm"]))
        out["candidates_ours"] = int(ours.size)
        out["candidates_common"] = len(ka & kb)
    return out


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    amps, N = make_spectrum()
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcsref.so")):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libcsref.so was not built (needs the reference sources)"}))
        return 0
    rates = []
    cores = 1
    sample = ""
    for _ in range(args.warmup):
        cpu_reference_rate(amps, N, seconds=0.5, max_reps=1)
    for _ in range(args.steps):
        r, cores, sample = cpu_reference_rate(amps, N, seconds=1.0, max_reps=4)
        rates.append(r)
    value = statistics.median(rates)
    from coherentsearch_c_b200.search import Options
    _, _, total = Options(blocksize=BLOCKSIZE_CPU).geometry(N, WORKLOAD["dt"])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": WORKLOAD,
        "blocksize": BLOCKSIZE_CPU,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_b200(args):
    import ctypes as C
    import numpy as np
    import torch
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    from coherentsearch_c_b200 import native as nt
    from coherentsearch_c_b200.search import Options, Session
    amps, N = make_spectrum()
    dt = WORKLOAD["dt"]
    opts = Options(nharms=60, m=16, blocksize=BLOCKSIZE_GPU, threshold=8.0)
    ses = Session(N, dt, opts, device=local)
    info = ses.info()
    total = ses.total
    gpu = nt.gpu_lib()

    # pinned host spectrum for the end-to-end arm
    pinned = torch.empty(amps.size, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = amps
    ft = nt.FFTFile()
    ft.amps = C.cast(C.c_void_p(pinned.data_ptr()), C.POINTER(C.c_float))
    ft.namps = amps.size // 2
    ft.N = N
    ft.T = N * dt
    ft.df = 1.0 / ft.T
    # device-resident spectrum: the session buffer, filled by one ABI run
    d_amps = ses.device_amps_ptr()
    ses.run_raw(amps)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step_device():
        ses.enqueue(d_amps)
        out, kms, rc = ses.collect()
        if rc == 1:                          # record buffer grown: redo
            ses.enqueue(d_amps)
            out, kms, rc = ses.collect()
        return out, kms

    for _ in range(args.warmup):
        step_device()
    stream = torch.cuda.current_stream()
    times, kernel_ms, ncand = [], [], 0
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out, kms = step_device()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            kernel_ms.append(kms)
            ncand = out.size
        torch.cuda.synchronize()
        # end-to-end through the reference ABI from pinned host memory
        e2e_times, nrec = [], 0
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cl = gpu.cs_gpu_session_run(ses.sess, C.byref(ft), opts.threshold)
            e1.record(stream)
            e1.synchronize()
            e2e_times.append(e0.elapsed_time(e1))
            nrec = int(cl.n)
            nt.host_lib().candlist_free(C.byref(cl))
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    ms = statistics.mean(times)
    kms = statistics.mean(kernel_ms)
    e2e_ms = statistics.mean(e2e_times)
    if pg is not None:
        t = torch.tensor([ms, kms, e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms, kms, e2e_ms = [float(v) for v in t.tolist()]
    value = world * total / (ms * 1e-3)
    e2e_value = world * total / (e2e_ms * 1e-3)
    hbm_peak, tc_peak, peak_kind = load_peaks()
    dft_tflops = total * DFT_FLOP_PER_TRIAL / (kms * 1e-3) / 1e12
    clocks = clk.summary()
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    simt_peak = 148 * 128 * f_sm
    simt_ach = total * SIMT_OPS_PER_TRIAL / (kms * 1e-3)
    kname = KERNEL_NAMES.get(info.kernel, "unknown")
    traffic = profiled_traffic(kname, total)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": WORKLOAD,
        "blocksize": BLOCKSIZE_GPU, "replicas": world,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(amps.nbytes),
                "d2h_bytes_per_step": int(nrec * 16 + 8)},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "tensor", "achieved": dft_tflops, "peak": tc_peak,
                     "unit": "TFLOP/s", "frac": dft_tflops / tc_peak, "traffic": traffic,
                     "kernel": kname, "kernel_ms": kms,
                     "peak_kind": f"bf16 dense, {peak_kind}",
                     "algorithmic": f"{DFT_FLOP_PER_TRIAL:.0f} DFT flop/trial x {total} trials"},
        "simt": {"achieved_lane_ops": simt_ach, "peak_lane_ops": simt_peak,
                 "frac": simt_ach / simt_peak, "ops_per_trial": SIMT_OPS_PER_TRIAL,
                 "note": "FP32 SIMT issue roofline at the sampled SM clock"},
        "clocks": clocks,
        "candidates": ncand,
        "session": {"tiles": info.ntiles, "chunks": info.nchunks, "grid": info.grid,
                    "smem_bytes": info.smem_bytes, "npad": info.npad, "kpad": info.kpad},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, cores, sample = cpu_reference_rate(amps, N, seconds=args.cpu_seconds)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores,
                                    "kind": "reference", "sample": sample,
                                    "cpu_model": cpu_model()}
            try:
                line["cpu_baseline"]["forms"] = cpu_reference_forms(amps, N)
            except Exception as exc:   # noqa: BLE001
                line["cpu_baseline"]["forms"] = {"unavailable": str(exc)}
        except Exception as exc:   # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0 and world == 1:
        try:
            line["precision"] = precision_study(ses, amps, N, dt, opts, local)
        except Exception as exc:   # noqa: BLE001
            line["precision"] = {"unavailable": str(exc)}
    if rank == 0 and world == 1:
        try:
            line["ducy"] = ducy_timing(ses, out, amps, N, dt)
        except Exception as exc:   # noqa: BLE001
            line["ducy"] = {"unavailable": str(exc)}
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        try:
            line["plain_reference_gpu"] = reference_gpu_rate(amps, N, dt, opts,
                                                             ours=ses.collapse(out))
        except Exception as exc:   # noqa: BLE001
            line["plain_reference_gpu"] = {"unavailable": str(exc)}
    if rank == 0 and world == 1 and not args.no_extras:
        # the batched and served forms in short (the sweep and serve workloads
        # have full lines of their own: --workload sweep / serve)
        try:
            lines, _ = sweep_lines(64, args.slots, [60], 1, 1, not args.no_ref_gpu, device=local)
            line["sweep"] = dict(lines[60], files=64,
                                 workload="64 spectra, lengths log-uniform 2^21-2^23 (dt 64 us), "
                                          "pulsar 11.2 Hz peaking mid-list, nharms 60; "
                                          f"{args.slots} batch slots; P1 = a session per file")
        except Exception as exc:   # noqa: BLE001
            line["sweep"] = {"unavailable": str(exc)}
        try:
            line["serve"] = serve_summary(400, 200.0, 24, args.slots, args.mem_budget_gb,
                                          not args.no_ref_gpu)
        except Exception as exc:   # noqa: BLE001
            line["serve"] = {"unavailable": str(exc)}
        # the raw-data front end's dedispersion (--workload dedisp has the full
        # line): 8-bit filterbank, 1024 channels x 2^22 spectra, 500 DMs
        for name, clipped in (("dedisp", False), ("dedisp_clipped", True)):
            try:
                line[name] = dedisp_summary(clipped, local)
            except Exception as exc:   # noqa: BLE001
                line[name] = {"unavailable": str(exc)}
    if rank == 0:
        print(json.dumps(line))
    ses.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


DEDISP = {
    "workload": "raw-data front end: 8-bit filterbank, 1024 channels, 1400 MHz centre, "
                "300 MHz, 64 us, 2^22 spectra, DM 56.8 pulsar; 64 subbands, 500 DMs 0-199.6 "
                "(step 0.4), SIGPROC blocks of 2400 spectra",
    "nchan": 1024, "nsub": 64, "ndm": 500, "lodm": 0.0, "dmstep": 0.4, "nspec": 1 << 22,
    "numout": 1 << 22,
}
DEDISP_METRIC = "dedispersed samples/sec/GPU"
DEDISP_UNIT = "DM-samples/s"


def make_filterbank_device(spec, device):
    """The synthetic filterbank of coherentsearch_c_b200.synth.make_filterbank,
    generated on the GPU (seeded torch generator) to keep set-up short."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(spec.seed)
    freqs = spec.lofreq + spec.chanwid * torch.arange(spec.nchan, device=device,
                                                      dtype=torch.float64)
    delay = spec.dm / (0.000241 * freqs * freqs)
    kappa = math.log(2.0) / (1.0 - math.cos(math.pi * spec.duty))
    raw = torch.empty((spec.nspec, spec.nchan), dtype=torch.uint8, device=device)
    chunk = 1 << 17
    for t0 in range(0, spec.nspec, chunk):
        n = min(chunk, spec.nspec - t0)
        t = (t0 + torch.arange(n, device=device, dtype=torch.float64))[:, None] * spec.dt
        phase = torch.remainder(spec.f0 * (t - delay[None, :]), 1.0)
        pulse = torch.exp(kappa * (torch.cos(2.0 * math.pi * phase) - 1.0)).float()
        x = spec.mean + spec.sigma * (torch.randn((n, spec.nchan), generator=g, device=device)
                                      + spec.amp * pulse)
        raw[t0:t0 + n] = torch.flip(torch.clamp(torch.round(x), 0, 255), dims=[1]).to(torch.uint8)
    return raw


def dedisp_cpu_rate(raw_host, t, seconds=10.0, clip_sigma=0.0):
    """The reference's dispersion.c kernels under the prepsubband block driver
    (oracle/_ref/libdedisp_ref.so, one thread, as prepsubband runs them) on a
    bounded stretch of the workload: all DMs over the first blocks; with
    clip_sigma > 0 its clip_times runs on every block first."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    nblk = 4 * t.blocks_per_read + 2
    sample = raw_host[: nblk * t.spectra_per_subint]
    reps, n_out, t0 = 0, 0, time.perf_counter()
    while True:
        out = rb.ref_dedisp_run(sample, t.nsub, t.idispdt, t.offsets, t.spectra_per_subint,
                                t.blocks_per_read, clip_sigma=clip_sigma)
        reps += 1
        n_out += out.shape[0] * out.shape[1]
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return n_out / dt, 1, (f"{reps} runs of all {t.ndm} DMs over the first {nblk} blocks "
                           f"({sample.shape[0]} spectra, {out.shape[1]} output samples per DM)")


def run_dedisp(args):
    world, rank, local, pg = dist_setup(args)
    line = dedisp_measure(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def dedisp_summary(clipped, local, steps=5, cpu_seconds=3.0):
    """The dedispersion workload in short for the search line: DM-samples/s,
    the two stages' kernel times, and the reference's CPU rate on a sample."""
    a = argparse.Namespace(clipped=clipped, nspec_log2=0, steps=steps, warmup=3,
                           no_e2e=True, no_cpu_baseline=False, cpu_seconds=cpu_seconds)
    line = dedisp_measure(a, 1, 0, local, None)
    out = {k: line[k] for k in ("value", "unit", "ms_per_step")}
    out["kernel"] = line["roofline"]["kernel"]
    out["subband_ms"] = line["roofline"]["subband_ms"]
    out["dm_ms"] = line["roofline"]["dm_ms"]
    out["hbm_frac"] = line["roofline"]["frac"]
    cb = line.get("cpu_baseline", {})
    out["cpu_baseline"] = cb
    if cb.get("value"):
        out["vs_cpu_baseline"] = line["value"] / cb["value"]
    if clipped:
        out["spectra_clipped"] = line["spectra_clipped"]
    return out


def dedisp_measure(args, world, rank, local, pg):
    import ctypes as C
    import torch
    from coherentsearch_c_b200 import synth
    from coherentsearch_c_b200.dedisp import Dedisperser, dedisp_tables
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    W = dict(DEDISP)
    if args.nspec_log2:
        W["nspec"] = W["numout"] = 1 << args.nspec_log2
        W["workload"] = W["workload"].replace("2^22 spectra", f"2^{args.nspec_log2} spectra")
    spec = synth.config_filterbank(nspec=W["nspec"], seed=4 + rank)
    t = dedisp_tables(W["nchan"], W["nsub"], W["ndm"], W["lodm"], W["dmstep"], spec.lofreq,
                      spec.chanwid, spec.dt)
    raw = make_filterbank_device(spec, dev)
    dd = Dedisperser(t, max_spectra=spec.nspec, device=local)
    nout = dd.output_length(spec.nspec, W["numout"])
    stride = (nout + 3) // 4 * 4
    out = torch.empty((t.ndm, stride), dtype=torch.float32, device=dev)
    # a stream of our own: the legacy default stream's handle is 0, which the
    # C ABI reads as "the plan's stream"
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    L = t.spectra_per_subint
    nclipped = 0
    if args.clipped:
        # RFI that the default 6-sigma clip replaces: every 64th block holds a
        # broadband burst of 4 spectra, every 97th a dropout spectrum
        nblk = spec.nspec // L
        for b in range(1, nblk, 64):
            raw[b * L + 100: b * L + 104] = 255
        for b in range(5, nblk, 97):
            raw[b * L + 7] = 0
        flags = torch.empty(nblk * L, dtype=torch.uint8, device=dev)
        levels = torch.empty(nblk * t.nchan, dtype=torch.float32, device=dev)
        scratch = torch.empty(dd.clip_scratch_bytes(spec.nspec), dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()

    def step():
        nonlocal nclipped
        if not args.clipped:
            return dd.run_device(raw.data_ptr(), spec.nspec, out.data_ptr(), stride,
                                 W["numout"], stream.cuda_stream)
        nclipped = dd.clip_levels(raw.data_ptr(), spec.nspec, flags.data_ptr(),
                                  levels.data_ptr(), 6.0, stream.cuda_stream,
                                  scratch.data_ptr(), scratch.numel())
        return dd.run_device_clipped(raw.data_ptr(), spec.nspec, flags.data_ptr(),
                                     levels.data_ptr(), out.data_ptr(), stride, W["numout"],
                                     stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    times, sb_ms, dm_ms = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            a, b = dd.last_times()
            sb_ms.append(a)
            dm_ms.append(b)
        torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    ms = statistics.mean(times)
    if pg is not None:
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms = float(tt.item())
    samples = t.ndm * nout
    value = world * samples / (ms * 1e-3)
    hbm_peak, _, peak_kind = load_peaks()
    alg_bytes = spec.nspec * t.nchan + 4.0 * samples          # raw once + output once
    kern_ms = statistics.mean(sb_ms) + statistics.mean(dm_ms)
    line = {
        "metric": DEDISP_METRIC, "value": value, "unit": DEDISP_UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8->f32",
        "data": "synthetic",
        "config": dict(workload=W["workload"] + (
                           "; prepsubband -clip 6 on RFI bursts (4 saturated spectra every 64 "
                           "blocks, a dropout every 97): clip decisions and levels, then the "
                           "clipped FP32 dedispersion" if args.clipped else ""),
                       output_per_dm=nout, blocks_per_read=t.blocks_per_read,
                       l2="inputs larger than L2 (raw input and output both > 126 MB)",
                       parallelism=f"replicas{world}"),
        "gpu_launches": (8 if args.clipped else 2) * args.steps,
        "roofline": {"bound": "hbm", "achieved": alg_bytes / (kern_ms * 1e-3) / 1e9,
                     "peak": hbm_peak, "unit": "GB/s",
                     "frac": alg_bytes / (kern_ms * 1e-3) / 1e9 / hbm_peak, "traffic": None,
                     "kernel": ("dd_subband_clip + dd_dms_f32" if args.clipped
                                else "dd_subband_u8 + dd_dms_u16"),
                     "subband_ms": statistics.mean(sb_ms), "dm_ms": statistics.mean(dm_ms),
                     "peak_kind": f"HBM copy, {peak_kind}",
                     "algorithmic": f"{spec.nspec} x {t.nchan} B raw + {samples} x 4 B output"},
        "clocks": clk.summary(),
    }
    if args.clipped:
        line["spectra_clipped"] = nclipped
        line["clip_levels_ms"] = ms - kern_ms
    # end to end: host (pinned) raw in, host (pinned) output back, through cs_dedisp_run
    if not args.no_e2e and not args.clipped:
        h_raw = torch.empty(raw.shape, dtype=torch.uint8, pin_memory=True)
        h_raw.copy_(raw)
        h_out = torch.empty((t.ndm, nout), dtype=torch.float32, pin_memory=True)
        e2e = []
        for _ in range(max(2, args.steps // 5)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            got = C.c_longlong(0)
            rc = dd.lib.cs_dedisp_run(dd.plan, h_raw.data_ptr(), spec.nspec, W["numout"],
                                      h_out.data_ptr(), nout, C.byref(got))
            e1.record(stream)
            e1.synchronize()
            if rc != 0:
                raise RuntimeError("cs_dedisp_run failed")
            e2e.append(e0.elapsed_time(e1))
        line["e2e"] = {"value": world * samples / (statistics.mean(e2e) * 1e-3),
                       "unit": DEDISP_UNIT, "h2d_bytes_per_step": int(h_raw.numel()),
                       "d2h_bytes_per_step": int(4 * samples)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            nblk = 4 * t.blocks_per_read + 2
            host = raw[: nblk * t.spectra_per_subint].cpu().numpy()
            rate, cores, sample = dedisp_cpu_rate(host, t, seconds=args.cpu_seconds,
                                                  clip_sigma=6.0 if args.clipped else 0.0)
            line["cpu_baseline"] = {"value": rate, "unit": DEDISP_UNIT, "cores": cores,
                                    "kind": "reference", "sample": sample}
        except Exception as exc:   # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": DEDISP_UNIT, "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {exc}"}
    dd.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return line


def prep_cpu_rate(series_host, dd_rate, N, dt, opts, seconds=10.0):
    """The reference CPU path of one DM on the host cores: its dedispersion
    cost per DM at the measured dispersion.c rate (one thread, as
    prepsubband runs it), plus realfft + rednoise and the OpenMP search of
    full-length dedispersed series, repeated for about `seconds`.  Returns
    (trials/s, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    cores = os.cpu_count() or 1
    rb.ref_lib()
    rb.pin_ref_threads(cores)
    _, _, total = opts.geometry(N, dt)
    reps, t0 = 0, time.perf_counter()
    while True:
        x = series_host[reps % len(series_host)]
        amps = rb.ref_spectrum(x, dt)
        rb.ref_search(amps, N, dt, opts)
        reps += 1
        if time.perf_counter() - t0 >= seconds or reps >= 8:
            break
    per_dm = (time.perf_counter() - t0) / reps + N / dd_rate
    return total / per_dm, cores, (f"{reps} DM series of {N} points: realfft + rednoise + search "
                                   f"(OpenMP, {cores} threads), plus {N} dedispersed samples "
                                   f"per DM at the reference dispersion rate {dd_rate:.3g}/s")


def run_prep(args):
    """Raw-data front end end to end on one GPU: 8-bit filterbank ->
    subband dedispersion (500 DMs) -> padding -> realfft + rednoise ->
    coherent search of every DM (nharms 60, m 16)."""
    import torch
    from coherentsearch_c_b200 import synth
    from coherentsearch_c_b200.dedisp import dedisp_tables
    from coherentsearch_c_b200.prep import PrepSearch
    from coherentsearch_c_b200.search import Options
    world, rank, local, pg = dist_setup(args)
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    W = dict(DEDISP)
    if args.nspec_log2:
        W["nspec"] = W["numout"] = 1 << args.nspec_log2
        W["workload"] = W["workload"].replace("2^22 spectra", f"2^{args.nspec_log2} spectra")
    if args.ndm:
        W["ndm"] = args.ndm
        W["workload"] = W["workload"].replace("500 DMs 0-199.6", f"{args.ndm} DMs from 0")
    spec = synth.config_filterbank(nspec=W["nspec"], seed=4 + rank)
    t = dedisp_tables(W["nchan"], W["nsub"], W["ndm"], W["lodm"], W["dmstep"], spec.lofreq,
                      spec.chanwid, spec.dt)
    opts = Options(nharms=60, m=16, blocksize=65536, threshold=8.0)
    raw = make_filterbank_device(spec, dev)
    ps = PrepSearch(t, spec.nspec, W["numout"], spec.dt, opts, device=local)
    N, total = ps.N, ps.ses.total
    stream = ps.stream

    def step():
        ps.dedisperse(raw.data_ptr(), spec.nspec)
        return ps.search_all(collapse=True)      # search_file's list per DM

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    times, dd_ms, search_ms, ncand = [], [], [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            a, b = ps.dd.last_times()
            dd_ms.append(a + b)
            search_ms.append(sum(ps.search_ms))
            ncand = sum(r.size for r in res)
        torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    ms = statistics.mean(times)
    if pg is not None:
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        ms = float(tt.item())
    trials = t.ndm * total
    value = world * trials / (ms * 1e-3)
    hbm_peak, tc_peak, peak_kind = load_peaks()
    kms = statistics.mean(search_ms)
    # the default 6-sigma clip decisions and channel levels, timed on their
    # own (they run inside each step, before the dedispersion)
    torch.cuda.synchronize()
    c0 = time.perf_counter()
    ps.dd.clip_levels(raw.data_ptr(), spec.nspec, ps._clip_flags.data_ptr(),
                      ps._clip_levels.data_ptr(), ps.clip_sigma, stream.cuda_stream,
                      ps._clip_scratch.data_ptr(), ps._clip_scratch.numel())
    clip_ms = 1e3 * (time.perf_counter() - c0)
    dft_tflops = trials * DFT_FLOP_PER_TRIAL / (kms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8->f32",
        "data": "synthetic",
        "config": dict(workload=W["workload"] + "; search of every DM: N=" + str(N)
                       + " (numout), nharms 60, m 16, hidr 0.5, 0.1-125 Hz, maxdecim 6, "
                       "blocksize 65536, threshold 8; each DM's candidates collapsed "
                       "(remove_duplicates + remove_harmonics) on the GPU",
                       ndm=t.ndm, trials_per_dm=total,
                       output_per_dm=ps.nout,
                       l2="inputs larger than L2 (raw input and dedispersed output > 126 MB)",
                       parallelism=f"replicas{world}"),
        # clip decisions and levels 6, dedispersion 2; per DM spectrum 4, search 2,
        # collapse 10 (cuFFT, CUB and PyTorch's fills not counted)
        "gpu_launches": (8 + 16 * t.ndm) * args.steps,
        "roofline": {"bound": "tensor", "achieved": dft_tflops, "peak": tc_peak,
                     "unit": "TFLOP/s", "frac": dft_tflops / tc_peak, "traffic": None,
                     "kernel": "search_ws_cfg60", "kernel_ms_per_dm": kms / t.ndm,
                     "peak_kind": f"bf16 dense, {peak_kind}",
                     "algorithmic": f"{DFT_FLOP_PER_TRIAL:.0f} DFT flop/trial x {total} trials "
                                    f"x {t.ndm} DMs"},
        "stages_ms": {"dedisp": statistics.mean(dd_ms), "search_kernels": kms,
                      "rest": ms - statistics.mean(dd_ms) - kms,
                      "clip_levels": clip_ms, "steps": [round(x, 2) for x in times]},
        "spectra_clipped": ps.nclipped,
        "clocks": clk.summary(),
        "candidates": ncand,
    }
    # end to end: pinned host filterbank in, every DM's candidates back
    if not args.no_e2e:
        h_raw = torch.empty(raw.shape, dtype=torch.uint8, pin_memory=True)
        h_raw.copy_(raw)
        e2e, nbytes_back = [], 0
        for _ in range(max(2, args.steps // 2)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                raw.copy_(h_raw, non_blocking=True)
            res = step()
            e1.record(stream)
            e1.synchronize()
            e2e.append(e0.elapsed_time(e1))
            nbytes_back = sum(r.nbytes for r in res)
        line["e2e"] = {"value": world * trials / (statistics.mean(e2e) * 1e-3), "unit": UNIT,
                       "h2d_bytes_per_step": int(h_raw.numel()),
                       "d2h_bytes_per_step": int(nbytes_back)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            nblk = 4 * t.blocks_per_read + 2
            host = raw[: nblk * t.spectra_per_subint].cpu().numpy()
            dd_rate, _, _ = dedisp_cpu_rate(host, t, seconds=max(2.0, args.cpu_seconds / 3))
            ser = [ps.series(d) for d in (0, t.ndm // 2)]
            rate, cores, sample = prep_cpu_rate(ser, dd_rate, N, spec.dt, opts,
                                                seconds=args.cpu_seconds)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores,
                                    "kind": "reference", "sample": sample}
        except Exception as exc:   # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0:
        print(json.dumps(line))
    ps.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def spectrum_device(N, dt, seed, pulsars, device):
    """A normalised spectrum as synth.normalised_spectrum builds it (white
    noise + von Mises pulse trains, PRESTO-packed forward FFT, unit power by
    block medians of 100 bins), computed on the GPU and returned in pinned
    host memory as interleaved float32 (a spectrum read from a file)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.randn(N, generator=g, device=device, dtype=torch.float64)
    t = torch.arange(N, device=device, dtype=torch.float64) * dt
    for p in pulsars:
        kappa = math.log(2.0) / (1.0 - math.cos(math.pi * p.duty))
        s = torch.exp(kappa * (torch.cos(2.0 * math.pi * torch.remainder(t * p.f0 + p.phase0, 1.0))
                               - 1.0))
        s = s - s.mean()
        x = x + (p.snr / torch.sqrt(torch.dot(s, s))) * s
    X = torch.fft.rfft(x)
    n2 = N // 2
    S = X[:n2].clone()
    pw = (S.real ** 2 + S.imag ** 2)
    nb = (n2 - 1) // 100
    scale = torch.ones(n2, device=device, dtype=torch.float64)
    if nb > 0:
        med = torch.quantile(pw[1:1 + nb * 100].reshape(nb, 100), 0.5, dim=1) / math.log(2.0)
        med[med <= 0] = 1.0
        scale[1:1 + nb * 100] = torch.repeat_interleave(1.0 / torch.sqrt(med), 100)
        scale[1 + nb * 100:] = 1.0 / torch.sqrt(med[-1])
    S = (S * scale).to(torch.complex64)
    S[0] = 1.0 + 0.0j
    out = torch.empty(2 * n2, dtype=torch.float32, pin_memory=True)
    out.copy_(torch.view_as_real(S).reshape(-1))
    return out


def _same_cands(a, b):
    return a.size == b.size and all(np.array_equal(a[f], b[f]) for f in ("r", "metric", "nharm"))


def sweep_reference_gpu(specs, spectra, dt, opts, trials, ours, batched_ms):
    """The reference's own GPU form over the same file list, one file at a
    time through its search_file with one SearchCache (it rebuilds the
    session whenever the length changes, src/search.c:1388-1406), raw
    candidates; host wall time."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    if not rb.have_ref_gpu():
        return {"unavailable": "oracle/_ref/libcsref_gpu.so not built"}
    srch = rb.RefGpuSearcher(opts)
    try:
        srch.search(spectra[0], specs[0].N, dt, collapse=False)     # warm
        t0 = time.perf_counter()
        out = [srch.search(a, sp.N, dt, collapse=False) for sp, a in zip(specs, spectra)]
        wall = time.perf_counter() - t0
    finally:
        srch.close()
    same = sum(1 for x, y in zip(out, ours)
               if set(zip(np.round(x["r"], 9), x["nharm"])) == set(zip(np.round(y["r"], 9), y["nharm"])))
    return {"ms": 1e3 * wall, "trials_per_s": trials / wall,
            "batched_vs_reference_gpu": 1e3 * wall / batched_ms,
            "files_with_identical_candidate_sets": same, "files": len(specs),
            "candidates": int(sum(o.size for o in out)),
            "source": "reference src/cuda.cu built for sm_100a, one SearchCache over the list"}


def sweep_lines(files, slots, nh_list, steps, warmup, ref_gpu, device=0):
    """Config 3 measured: `files` spectra of uneven length searched plain (P1:
    a session per file, this library's single-file form), batched
    (cs_gpu_batch: slots, one launch per file) and grouped (sweep.search_list:
    one persistent launch per group of files, group size from the autotuner
    on the first 64 files), optionally beside the reference's own GPU form
    (P0), per harmonic count.  Returns ({nh: summary}, spectra)."""
    import torch
    from coherentsearch_c_b200 import synth
    from coherentsearch_c_b200.batch import Batch
    from coherentsearch_c_b200 import native as nt
    from coherentsearch_c_b200.search import MultiGraph, Options, Session, multi_search
    from coherentsearch_c_b200.sweep import autotune, search_list, warm
    specs = synth.config_dm_sweep(n_files=files)
    dt = specs[0].dt
    pinned = [spectrum_device(sp.N, dt, sp.seed, sp.pulsars, f"cuda:{device}") for sp in specs]
    spectra = [p.numpy() for p in pinned]
    listed = [(sp.N, None) for sp in specs]
    # device buffers of the grouped form, allocated before any timing; the
    # copies into them run inside the timed region
    dev_bufs = [torch.empty(p.numel(), dtype=torch.float32, device=f"cuda:{device}")
                for p in pinned]

    def upload(i):
        """Spectrum i to the device on the current stream (pinned source, so
        the copy overlaps the previous group's kernel)."""
        dev_bufs[i].copy_(pinned[i], non_blocking=True)
        return dev_bufs[i].data_ptr()
    lines = {}
    for nh in nh_list:
        opts = Options(nharms=nh, blocksize=65536, threshold=8.0)
        trials = sum(int(opts.geometry(sp.N, dt)[2]) for sp in specs)

        def plain():
            out = []
            for sp, a in zip(specs, spectra):
                ses = Session(sp.N, dt, opts)
                out.append(ses.run_raw(a))
                ses.close()
            return out

        # a long-lived engine, as a serving process keeps one: created and its
        # slots loaded for the longest file before the timed region
        engine = Batch(nslots=slots)
        engine.warm(max(sp.N for sp in specs), dt, opts)

        def batched():
            ids = [engine.submit(a, sp.N, dt, opts) for sp, a in zip(specs, spectra)]
            return [engine.wait(i)[0] for i in ids]

        st = torch.cuda.current_stream().cuda_stream
        warm(max(sp.N for sp in specs), dt, opts, 64, device)   # two groups of up to 32
        group, tune = autotune(listed, dt, opts, candidates=(1, 2, 4, 8, 16, 32), sample=64,
                               device=device, upload=upload, stream=st,
                               sync=torch.cuda.synchronize)

        def grouped():
            return search_list(listed, dt, opts, group, device, upload, st)

        for _ in range(warmup):           # warm: modules, allocator, page cache
            for i in [engine.submit(a, sp.N, dt, opts) for sp, a in zip(specs[:4], spectra[:4])]:
                engine.wait(i)
        stream = torch.cuda.current_stream()
        res = {}
        for name, fn in (("plain", plain), ("batched", batched), ("grouped", grouped)):
            ts = []
            for _ in range(max(1, min(steps, 2))):
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                out = fn()
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            res[name] = (statistics.mean(ts), out)
        engine.close()
        # every spectrum resident on the device, searched by ONE persistent
        # launch over all their tiles (the kernel-side bound of the grouped form)
        for i in range(len(specs)):
            upload(i)
        resident = [Session(sp.N, dt, opts, device=device) for sp in specs]
        ptrs = [b.data_ptr() for b in dev_bufs]
        try:
            multi_search(resident, ptrs, stream=st)                # warm
            rts, rks = [], []
            for _ in range(max(1, min(steps, 2))):
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rout, kms = multi_search(resident, ptrs, stream=st)
                e1.record(stream)
                e1.synchronize()
                rts.append(e0.elapsed_time(e1))
                rks.append(kms)
            # the same launch recorded once as a CUDA graph and replayed
            graph = MultiGraph(resident, ptrs)
            try:
                graph.search(stream=st)                            # warm
                gts = []
                for _ in range(max(1, min(steps, 2))):
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    gout, _ = graph.search(stream=st)
                    e1.record(stream)
                    e1.synchronize()
                    gts.append(e0.elapsed_time(e1))
            finally:
                graph.close()
        finally:
            for ses in resident:
                ses.close()
            nt.gpu_lib().cs_b200_session_park_drain()
        diff = [i for i, (x, y) in enumerate(zip(res["plain"][1], res["batched"][1]))
                if not _same_cands(x, y)]
        equal = not diff
        lines[nh] = {"trials": trials, "plain_ms": res["plain"][0], "batched_ms": res["batched"][0],
                     "plain_trials_per_s": trials / (res["plain"][0] * 1e-3),
                     "batched_trials_per_s": trials / (res["batched"][0] * 1e-3),
                     "batched_vs_plain": res["plain"][0] / res["batched"][0],
                     "grouped_ms": res["grouped"][0],
                     "grouped_trials_per_s": trials / (res["grouped"][0] * 1e-3),
                     "grouped_vs_plain": res["plain"][0] / res["grouped"][0],
                     "grouped_files_per_launch": group,
                     "autotune_seconds_by_group": {str(k): v for k, v in tune.items()},
                     "grouped_equal_candidates": bool(all(
                         _same_cands(x, y) for x, y in zip(res["grouped"][1], res["plain"][1]))),
                     "resident_one_launch_ms": statistics.mean(rts),
                     "resident_one_launch_trials_per_s": trials / (statistics.mean(rts) * 1e-3),
                     "resident_one_launch_kernel_ms": statistics.mean(rks),
                     "resident_equal_candidates": bool(all(
                         _same_cands(x, y) for x, y in zip(rout, res["plain"][1]))),
                     "resident_graph_ms": statistics.mean(gts),
                     "resident_graph_trials_per_s": trials / (statistics.mean(gts) * 1e-3),
                     "resident_graph_equal_candidates": bool(all(
                         _same_cands(x, y) for x, y in zip(gout, res["plain"][1]))),
                     "equal_candidates": bool(equal), "differing_files": diff,
                     "candidates": int(sum(o.size for o in res["batched"][1])),
                     "plain_candidates": int(sum(o.size for o in res["plain"][1]))}
        if ref_gpu:
            lines[nh]["plain_reference_gpu"] = sweep_reference_gpu(
                specs, spectra, dt, opts, trials, res["batched"][1], res["batched"][0])
    return lines, spectra


def run_sweep(args):
    """Config 3: 256 files of uneven length.  `value`: every spectrum resident
    in HBM, one persistent launch over all their tiles; `e2e`: the grouped
    list driver (sweep.search_list, group size from its autotuner), spectra
    uploaded from pinned host memory inside the timed region.  The plain
    (a session per file) and batched (cs_gpu_batch) forms ride along."""
    import torch
    torch.cuda.set_device(0)
    lines, spectra = sweep_lines(args.files, args.slots, [60, 32], args.steps, args.warmup,
                                 not args.no_ref_gpu)
    h2d = int(sum(a.nbytes for a in spectra))
    main = lines[60]
    ngroups = -(-args.files // main["grouped_files_per_launch"])
    line = {
        "metric": METRIC, "value": main["resident_one_launch_trials_per_s"], "unit": UNIT,
        "n_gpus": 1, "steps": max(1, min(args.steps, 2)), "warmup": args.warmup,
        "ms_per_step": main["resident_one_launch_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"DM sweep: {args.files} spectra, lengths log-uniform "
                               "2^21-2^23 (dt 64 us), pulsar 11.2 Hz peaking mid-list; "
                               "nharms 60, m 16, blocksize 65536",
                   "inputs": "value: resident in HBM, one launch over all files; e2e: pinned "
                             "host memory, uploaded inside the timed region",
                   "l2": "inputs larger than L2 in aggregate", "parallelism": "replicas1"},
        "e2e": {"value": main["grouped_trials_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16 * main["candidates"]},
        # one amplitude-maximum kernel per file and one search kernel per group
        "gpu_launches": args.files + ngroups,
        "sweep": {str(k): v for k, v in lines.items()},
    }
    print(json.dumps(line))
    return 0


def serve_requests(nreq, npool, device=0):
    """Config 5's requests: a pool of seeded spectra (N log-uniform 2^20-2^24,
    30 % with a pulsar) and `nreq` requests drawn from it with nharms uniform
    in {16, 32, 60}."""
    from coherentsearch_c_b200 import synth
    from coherentsearch_c_b200.search import Options
    from coherentsearch_c_b200.serve import Request, log_uniform_lengths
    rng = np.random.default_rng(7)
    dt = 64e-6
    lengths = log_uniform_lengths(npool, 1 << 20, 1 << 24, seed=11)
    pool = []
    for i, N in enumerate(lengths):
        pulsars = []
        if rng.random() < 0.3:
            pulsars = [synth.Pulsar(float(math.exp(rng.uniform(math.log(0.5), math.log(100.0)))),
                                    float(rng.uniform(0.02, 0.10)), float(rng.uniform(8, 30)))]
        pool.append((N, spectrum_device(N, dt, 5000 + i, pulsars, f"cuda:{device}").numpy()))
    reqs = []
    for i in range(nreq):
        N, a = pool[int(rng.integers(npool))]
        nh = int(rng.choice([16, 32, 60]))
        reqs.append(Request(a, N, dt, Options(nharms=nh, blocksize=65536, threshold=8.0)))
    return reqs, max(lengths)


def serve_capacity(reqs, maxlen, slots, budget_gb):
    """Closed loop: every request submitted at once, served (continuous
    batching) and plain (a session per request).  The served throughput is
    the capacity of the engine; p50/p99 are latencies under saturation."""
    from coherentsearch_c_b200.search import Options
    from coherentsearch_c_b200.serve import PlainServer, SearchServer, run_stream
    zero = np.zeros(len(reqs))
    with SearchServer(nslots=slots, mem_budget=budget_gb << 30) as srv:
        srv.warm(maxlen, 64e-6, Options(nharms=60, blocksize=65536, threshold=8.0))
        served = run_stream(srv, reqs, zero)
    with PlainServer() as pl:
        plain = run_stream(pl, reqs, zero)
    return {"requests": len(reqs), "served_trials_per_s": served["trials_per_s"],
            "served_requests_per_s": len(reqs) / served["wall_s"],
            "served_p50_ms": served["p50_ms"], "served_p99_ms": served["p99_ms"],
            "plain_trials_per_s": plain["trials_per_s"],
            "plain_requests_per_s": len(reqs) / plain["wall_s"],
            "served_vs_plain": served["trials_per_s"] / plain["trials_per_s"],
            "equal_candidates": bool(all(_same_cands(x, y) for x, y in
                                         zip(served["results"], plain["results"])))}


def serve_load_curve(reqs, maxlen, slots, budget_gb, rates=(200, 400, 600, 800)):
    """Latency against offered load: the same requests as open-loop Poisson
    streams at each rate, through one engine loaded for the largest request.
    Past the capacity the queue grows for the whole stream and p99 with it."""
    from coherentsearch_c_b200.search import Options
    from coherentsearch_c_b200.serve import SearchServer, poisson_arrivals, run_stream
    curve = []
    with SearchServer(nslots=slots, mem_budget=budget_gb << 30) as srv:
        srv.warm(maxlen, 64e-6, Options(nharms=60, blocksize=65536, threshold=8.0))
        for rate in rates:
            res = run_stream(srv, reqs, poisson_arrivals(len(reqs), rate=rate, seed=3))
            curve.append({"offered_per_s": rate, "p50_ms": res["p50_ms"],
                          "p99_ms": res["p99_ms"], "trials_per_s": res["trials_per_s"],
                          "requests_per_s": len(reqs) / res["wall_s"]})
    return curve


def serve_summary(nreq, rate, npool, slots, budget_gb, ref_gpu):
    """Config 5 in short: an open-loop Poisson stream at `rate` (served and
    plain, p50/p99 from arrival to result), then the closed-loop capacity of
    both forms on the same requests, and the reference's own GPU form (P0)
    back to back on the first requests."""
    from coherentsearch_c_b200.search import Options
    from coherentsearch_c_b200.serve import (PlainServer, SearchServer, poisson_arrivals,
                                             run_stream)
    reqs, maxlen = serve_requests(nreq, npool)
    arrivals = poisson_arrivals(len(reqs), rate=rate, seed=3)
    with SearchServer(nslots=slots) as srv:              # warm both forms
        run_stream(srv, reqs[:6], np.zeros(6))
    with PlainServer() as pl:
        run_stream(pl, reqs[:3], np.zeros(3))
    with SearchServer(nslots=slots, mem_budget=budget_gb << 30) as srv:
        srv.warm(maxlen, 64e-6, Options(nharms=60, blocksize=65536, threshold=8.0))
        served = run_stream(srv, reqs, arrivals)
    with PlainServer() as pl:
        plain = run_stream(pl, reqs, arrivals)
    out = {"workload": f"{len(reqs)} requests, Poisson {rate}/s, N log-uniform 2^20-2^24, "
                       f"nharms in {{16, 32, 60}}, 30% with a pulsar (pool of {npool}); "
                       f"{slots} slots",
           "open_loop": {"served_p50_ms": served["p50_ms"], "served_p99_ms": served["p99_ms"],
                         "served_trials_per_s": served["trials_per_s"],
                         "plain_p50_ms": plain["p50_ms"], "plain_p99_ms": plain["p99_ms"],
                         "plain_trials_per_s": plain["trials_per_s"],
                         "equal_candidates": bool(all(_same_cands(x, y) for x, y in
                                                      zip(served["results"],
                                                          plain["results"])))},
           "closed_loop": serve_capacity(reqs, maxlen, slots, budget_gb),
           "load_curve": serve_load_curve(reqs, maxlen, slots, budget_gb)}
    if ref_gpu:
        p0 = serve_reference_gpu(reqs, served["results"], served["trials_per_s"], limit=30)
        out["plain_reference_gpu"] = p0
        rate0 = p0.get("trials_per_s") if isinstance(p0, dict) else None
        if rate0:
            out["closed_loop"]["served_vs_reference_gpu"] = (
                out["closed_loop"]["served_trials_per_s"] / rate0)
    return out


def run_serve(args):
    """Config 5: a Poisson stream of search requests served by the request
    loop (continuous batching) and by the plain per-request form."""
    import torch
    from coherentsearch_c_b200.search import Options
    from coherentsearch_c_b200.serve import (PlainServer, SearchServer, poisson_arrivals,
                                             run_stream)
    torch.cuda.set_device(0)
    dt = 64e-6
    npool = args.pool
    reqs, maxlen = serve_requests(args.requests, npool)
    lengths = [maxlen]
    arrivals = poisson_arrivals(len(reqs), rate=args.rate, seed=3)
    # warm both forms on a few requests
    with SearchServer(nslots=args.slots) as srv:
        run_stream(srv, reqs[:6], np.zeros(6))
    with PlainServer() as pl:
        run_stream(pl, reqs[:3], np.zeros(3))
    with ClockSampler(0) as clk:
        with SearchServer(nslots=args.slots, mem_budget=args.mem_budget_gb << 30) as srv:
            srv.warm(max(lengths), dt, Options(nharms=60, blocksize=65536, threshold=8.0))
            served = run_stream(srv, reqs, arrivals)
            qr = np.array(srv.stats) if srv.stats else np.zeros((1, 2))
            held = srv.batch.device_bytes()
    with PlainServer() as pl:
        plain = run_stream(pl, reqs, arrivals)
    equal = all(_same_cands(x, y) for x, y in zip(served["results"], plain["results"]))
    trials = served["trials"]
    line = {
        "metric": METRIC, "value": served["trials_per_s"], "unit": UNIT, "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * served["wall_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"serving stream: {len(reqs)} requests, Poisson {args.rate}/s, "
                               "N log-uniform 2^20-2^24, nharms in {16, 32, 60}, 30% with a "
                               f"pulsar (spectra from a pool of {npool}); {args.slots} slots, "
                               f"{args.mem_budget_gb} GB budget, slots loaded for the "
                               "largest request before the stream",
                   "inputs": "pinned host memory, uploaded per request",
                   "parallelism": "replicas1"},
        "latency_ms": {"p50": served["p50_ms"], "p99": served["p99_ms"], "mean": served["mean_ms"],
                       "queued_p50": float(np.percentile(qr[:, 0], 50)),
                       "queued_p99": float(np.percentile(qr[:, 0], 99)),
                       "on_slot_p50": float(np.percentile(qr[:, 1], 50)),
                       "on_slot_p99": float(np.percentile(qr[:, 1], 99)),
                       "on_slot_max": float(qr[:, 1].max())},
        "plain": {"trials_per_s": plain["trials_per_s"], "p50_ms": plain["p50_ms"],
                  "p99_ms": plain["p99_ms"], "mean_ms": plain["mean_ms"],
                  "wall_s": plain["wall_s"]},
        "served_vs_plain": served["trials_per_s"] / plain["trials_per_s"],
        "device_bytes_held": held,
        "equal_candidates": bool(equal), "trials": trials,
        "e2e": {"value": served["trials_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": int(sum(r.amps.nbytes for r in reqs)),
                "d2h_bytes_per_step": int(16 * sum(x.size for x in served["results"]))},
        "gpu_launches": 2 * len(reqs),
        "clocks": clk.summary(),
    }
    line["load_curve"] = serve_load_curve(reqs, maxlen, args.slots, args.mem_budget_gb)
    if not args.no_ref_gpu:
        line["plain_reference_gpu"] = serve_reference_gpu(reqs, served["results"],
                                                          served["trials_per_s"])
    print(json.dumps(line))
    return 0


def serve_reference_gpu(reqs, served_results, served_rate, limit=60):
    """The reference's own GPU form serving the first `limit` requests back to
    back (no arrival gaps, so it is not idle): its search_file with a session
    per request, raw candidates; host wall time."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind as rb
    if not rb.have_ref_gpu():
        return {"unavailable": "oracle/_ref/libcsref_gpu.so not built"}
    sub = reqs[:limit]
    rb.ref_search_gpu(sub[0].amps, sub[0].N, sub[0].dt, sub[0].opts, collapse=False)  # warm
    t0 = time.perf_counter()
    out = [rb.ref_search_gpu(r.amps, r.N, r.dt, r.opts, collapse=False) for r in sub]
    wall = time.perf_counter() - t0
    trials = sum(r.trials for r in sub)
    same = sum(1 for x, y in zip(out, served_results)
               if set(zip(np.round(x["r"], 9), x["nharm"])) == set(zip(np.round(y["r"], 9), y["nharm"])))
    return {"requests": len(sub), "trials_per_s": trials / wall, "mean_ms": 1e3 * wall / len(sub),
            "served_vs_reference_gpu": served_rate / (trials / wall),
            "requests_with_identical_candidate_sets": same,
            "source": "reference src/cuda.cu built for sm_100a, search_file per request, "
                      "requests back to back (a lower bound on its latency under load)"}


def run_series(args):
    """The small configuration end to end: an N = 2^20 float32 series (7.3 Hz
    pulsar, 5 % duty) -> realfft + rednoise on the GPU -> search (nharms 60,
    m 16, blocksize 2048, threshold 8) -> search_file's collapsed list."""
    import torch
    from coherentsearch_c_b200 import synth
    from coherentsearch_c_b200.search import Options, Session
    from coherentsearch_c_b200.spectrum import SpectrumMaker
    torch.cuda.set_device(0)
    dev = "cuda:0"
    spec = synth.config_small()
    x = synth.make_series(spec).astype(np.float32)
    N, dt = x.size, spec.dt
    opts = Options(nharms=60, m=16, blocksize=2048, threshold=8.0)
    ses = Session(N, dt, opts)
    sm = SpectrumMaker(N, dt)
    total = ses.total
    stream = torch.cuda.Stream(device=dev)
    d_x = torch.from_numpy(x).to(dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def step():
        sm.run_device(d_x.data_ptr(), ses.device_amps_ptr(), stream.cuda_stream)
        ses.enqueue(None, after_stream=stream.cuda_stream)
        out, kms, rc = ses.collect_collapsed()
        if rc == 1:
            ses.enqueue(None)
            out, kms, rc = ses.collect_collapsed()
        return out, kms

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times, kern = [], []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out, kms = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            kern.append(kms)
        # end to end: the series from pinned host memory, candidates back
        h_x = torch.empty(N, dtype=torch.float32, pin_memory=True)
        h_x.numpy()[:] = x
        e2e = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                d_x.copy_(h_x, non_blocking=True)
            out, _ = step()
            e1.record(stream)
            e1.synchronize()
            e2e.append(e0.elapsed_time(e1))
    ms = statistics.mean(times)
    kms = statistics.mean(kern)
    hbm_peak, tc_peak, peak_kind = load_peaks()
    dft = total * DFT_FLOP_PER_TRIAL / (kms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": total / (ms * 1e-3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "small configuration: N=2^20 f32 series, dt 64 us, 7.3 Hz "
                               "pulsar (5 % duty, folded S/N ~15) in white noise; realfft + "
                               "rednoise on the GPU, search nharms 60, m 16, blocksize 2048, "
                               "lobin 100, 0.1-125 Hz, hidr 0.5, threshold 8, collapsed",
                   "trials": total, "l2": "flushed (512 MiB write) before each timed step",
                   "parallelism": "replicas1"},
        "e2e": {"value": total / (statistics.mean(e2e) * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": int(x.nbytes), "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": 16 * args.steps,     # 4 spectrum, 2 search, 10 collapse (cuFFT, CUB not counted)
        "roofline": {"bound": "tensor", "achieved": dft, "peak": tc_peak, "unit": "TFLOP/s",
                     "frac": dft / tc_peak, "traffic": None,
                     "kernel": KERNEL_NAMES.get(ses.info().kernel, "unknown"),
                     "kernel_ms": kms, "peak_kind": f"bf16 dense, {peak_kind}"},
        "candidates": int(out.size),
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import refbind as rb
        cores = os.cpu_count() or 1
        rb.ref_lib()
        rb.pin_ref_threads(cores)
        ref = rb.ref_search(rb.ref_spectrum(x, dt), N, dt, opts)
        reps, t0 = 0, time.perf_counter()
        while reps < 40:
            rb.ref_search(rb.ref_spectrum(x, dt), N, dt, opts)
            reps += 1
            if time.perf_counter() - t0 >= args.cpu_seconds:
                break
        rate = total * reps / (time.perf_counter() - t0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                                "sample": f"{reps} runs of realfft + rednoise + search_file "
                                          f"(OpenMP, {cores} threads) on the same series"}
        line["candidates_reference"] = int(ref.size)
        line["candidates_common"] = len(set(zip(np.round(ref["r"], 9), ref["nharm"])) &
                                        set(zip(np.round(out["r"], 9), out["nharm"])))
    print(json.dumps(line))
    ses.close()
    sm.close()
    return 0


def profiled_traffic(kernel, total):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary profiles/<kernel>_n23_traffic.md, a line `bytes_per_launch: B`
    measured on this workload (same trial count), else None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_n23_traffic.md")
    if not os.path.exists(path):
        return None
    vals = {}
    for line in open(path):
        line = line.strip().strip("`")
        if ":" in line:
            k, _, v = line.partition(":")
            vals[k.strip()] = v.strip().replace(",", "")
    try:
        if int(vals.get("trials", -1)) != total:
            return None
        return int(vals["bytes_per_launch"])
    except (KeyError, ValueError):
        return None


def main():
    # the grouped sweep keeps two groups of sessions (up to 2 x 32) in the
    # library's session park between groups
    os.environ.setdefault("CS_B200_SESSION_PARK", "80")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="search",
                    choices=["search", "dedisp", "sweep", "serve", "prep", "series"],
                    help="search: the coherent search (headline); dedisp: subband "
                         "dedispersion of the 8-bit filterbank workload; sweep: batched "
                         "search of a list of uneven-length files; serve: a Poisson "
                         "stream of requests through the request loop; prep: the raw-data "
                         "front end, filterbank -> dedispersion -> search of every DM; "
                         "series: the small configuration from a time series")
    ap.add_argument("--files", type=int, default=256, help="sweep: number of files")
    ap.add_argument("--slots", type=int, default=3, help="sweep/serve: batch slots")
    ap.add_argument("--requests", type=int, default=800, help="serve: requests")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    ap.add_argument("--pool", type=int, default=48, help="serve: distinct spectra")
    ap.add_argument("--mem-budget-gb", type=int, default=24, help="serve: device budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="search: skip the short sweep and serve summaries")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference's own GPU form (plain single-file baseline)")
    ap.add_argument("--clipped", action="store_true",
                    help="dedisp: RFI bursts and prepsubband's -clip 6 path")
    ap.add_argument("--nspec-log2", type=int, default=0,
                    help="dedisp workload length 2^n spectra (default: the 2^22 workload; "
                         "smaller sizes are for profiling captures only)")
    ap.add_argument("--ndm", type=int, default=0,
                    help="prep: DM trials (default: the 500-DM workload; fewer for profiling)")
    ap.add_argument("--nlog2", type=int, default=23,
                    help="series length 2^n (23 = the benchmark workload; smaller "
                         "sizes are for profiling captures only)")
    args = ap.parse_args()
    if args.nlog2 != 23:
        WORKLOAD["N"] = 1 << args.nlog2
        WORKLOAD["workload"] = WORKLOAD["workload"].replace("N=2^23", f"N=2^{args.nlog2}")
    if args.warmup < 3:
        args.warmup = 3
    if args.workload in ("sweep", "serve"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "this workload's baseline is its plain-form object"}))
            return 0
        return run_sweep(args) if args.workload == "sweep" else run_serve(args)
    if args.workload == "dedisp":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the dedispersion workload's reference arm is the cpu_baseline "
                              "object of its own line"}))
            return 0
        return run_dedisp(args)
    if args.workload == "series":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the small configuration's reference arm is the cpu_baseline "
                              "object of its own line"}))
            return 0
        return run_series(args)
    if args.workload == "prep":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the front-end workload's reference arm is the cpu_baseline "
                              "object of its own line"}))
            return 0
        return run_prep(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
