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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "precision-study single file: N=2^23 f32 series, dt=64us, nharms=60, m=16, "
                "hidr=0.5, 0.1-125 Hz, maxdecim 6, blocksize 65536, threshold 8",
    "N": 1 << 23, "dt": 64e-6, "nharms": 60, "m": 16, "blocksize": 65536,
    "l2": "flushed (512 MiB write) before each timed step",
}
METRIC = "Fourier trials/sec/GPU"
UNIT = "trials/s"
DFT_FLOP_PER_TRIAL = 28560.0      # 2*(2nh-1)*2nh at nh=60 (k | nh folds add none)
SIMT_OPS_PER_TRIAL = 6000.0       # interp 1920 FMA + 360 rotate + boxcar/fold ~3700


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
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

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
    opts = Options(blocksize=2048, threshold=8.0)
    _, _, total = opts.geometry(N, WORKLOAD["dt"])
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
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
              f"with the reference CPU path (blocksize 2048, its CPU default)")
    return total * reps / dt, cores, sample


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
    _, _, total = Options(blocksize=2048).geometry(N, WORKLOAD["dt"])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": WORKLOAD,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
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
    opts = Options(nharms=60, m=16, blocksize=WORKLOAD["blocksize"], threshold=8.0)
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
    kname = "search_ws60" if info.kernel == 1 else "cs_search_kernel"
    traffic = profiled_traffic(kname, total)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": dict(WORKLOAD, parallelism=f"replicas{world}"),
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
                                    "kind": "reference", "sample": sample}
        except Exception as exc:   # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0:
        print(json.dumps(line))
    ses.close()
    if pg is not None:
        pg.destroy_process_group()
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
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nlog2", type=int, default=23,
                    help="series length 2^n (23 = the benchmark workload; smaller "
                         "sizes are for profiling captures only)")
    args = ap.parse_args()
    if args.nlog2 != 23:
        WORKLOAD["N"] = 1 << args.nlog2
        WORKLOAD["workload"] = WORKLOAD["workload"].replace("N=2^23", f"N=2^{args.nlog2}")
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
