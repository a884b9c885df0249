"""Benchmark: 3D complex-to-complex FFT, forward then inverse (1/N), on B200.

Workload (the headline): 256 x 256 x 256 complex128 (f64 high_accuracy plan),
entries i.i.d. standard normal re/im from a seed, forward then normalized
inverse per step.  Inputs (268 MB) exceed the 126 MB L2, so no flush is needed
between steps.  Every other measured configuration is timed in the same run and
reported under "also", each with its error against the oracle: the other C2
shapes and dtypes (243x250x343, complex64), C1 (64 x 4096 f64), C3 (4096
uneven complex64 lengths), C4 (16384 x 4096 complex64: FP32 and the
split-precision tensor-core forms) and C5 (8 x 2048^2 real f32 with gradient).

value        : whole-job GFLOP/s, 5 N log2 N per transform, two transforms per step,
               data already in HBM, CUDA events on the launching stream.
roofline     : algorithmic bytes (2 N sizeof(complex) per transform; intermediate
               passes not counted) over the measured time, against the measured
               copy bandwidth in MEASURED_PEAKS.json.  Per launch this is the
               transform's bytes split over its launches; `per_pass_frac` is the
               separate figure of one pass's own read + write of the volume.
e2e          : the same metric through afc_execute_host (the reference-facing slice
               API) from pinned host buffers, copies inside the timed region; the
               measured pinned copy bandwidth of the host link is reported beside it.
cpu_baseline : the oracle's restatement of the reference CPU plan (FftPlan3D<f64>),
               all host threads, one forward+inverse of the same volume.

--impl reference times that CPU path alone on the same config, with a live
calibration of the restatement against the reference's published single-thread
latencies.  Multi-GPU: replicas only (one transform per rank, no collective on
the data path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (256, 256, 256)
ALSO = [((243, 250, 343), "f64"), ((256, 256, 256), "f32"), ((243, 250, 343), "f32")]
# the reference's published single-thread forward latencies (ns) of its 1D plans:
# benchmark_results.md:74,138,211,212 (criterion, clone-inclusive) and the
# checklist.md:1689-1699 / 1622-1624 dev-log N=4096 figures
PUBLISHED_NS = {("f64", 64): 147.20, ("f64", 128): 322.56, ("f64", 4096): 15844.0, ("f64", 10007): 494364.58,
                ("f64", 32768): 185739.87, ("f32", 64): 97.97, ("f32", 128): 177.00, ("f32", 4096): 5429.8,
                ("f32", 10007): 365107.41, ("f32", 32768): 134409.78}
METRIC = "FFT GFLOP/s (5N log2N) and % HBM roofline vs plain FP32, at stated FP64-oracle error"


def flops_per_transform(shape):
    n = int(np.prod(shape))
    return 5.0 * n * math.log2(n)


def bytes_per_transform(shape, prec):
    return 2.0 * int(np.prod(shape)) * (16 if prec == "f64" else 8)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl" if os.environ.get("AFC_BENCH_BACKEND", "nccl") == "nccl" else "gloo",
                                timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(v: float, world: int, device) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region.

    NVML is polled about every millisecond from a thread (a timed region of a
    few milliseconds still gets samples; nvidia-smi's loop cannot go below a
    few hundred milliseconds).  Only samples taken between `start()` and
    `stop()` count.  Falls back to an `nvidia-smi -lms 200` loop when NVML is
    unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []  # (sm_mhz, reason bits)
        self.max_mhz = None
        self.active = False
        self.done = False
        self.nv = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            self.nv, self.h = self._handle()
            nv = self.nv
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self.get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _poll(self):
        nv = self.nv
        while not self.done:
            if self.active:
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                                         int(self.get_reasons(self.h))))
                except Exception:
                    pass
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            if self.active:
                self.lines.append(line.strip())

    def start(self):
        self.active = True

    def stop(self):
        self.active = False

    def __exit__(self, *a):
        self.done = True
        self.active = False
        if self.nv is not None:
            self.t.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        for mhz, bits in self.samples:
            sm.append(mhz)
            for nm, b in self.REASONS.items():
                if bits & b:
                    reasons.add(nm)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def c2_input(shape, seed=2):
    """re/im i.i.d. N(0,1) from a seed (the C2 configuration's input)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def c2_config(shape, prec, world):
    """The config dict both arms print (same keys and values)."""
    nbytes = int(np.prod(shape)) * (16 if prec == "f64" else 8)
    return {"workload": f"3D C2C {'x'.join(map(str, shape))} {'complex128' if prec == 'f64' else 'complex64'}"
                        " forward+inverse (1/N)", "shape": list(shape),
            "precision": "f64 high_accuracy" if prec == "f64" else "f32 low_precision",
            "parallelism": f"replicas x{world}",
            "l2": f"inputs ({nbytes / 1e6:.0f} MB) larger than L2; no flush"}


def cpu_transform_gflops(shape, reps, threads=0, x=None):
    """Oracle FftPlan3D<f64> forward + inverse on host cores.  Returns
    (GFLOP/s, seconds, forward output of the last rep)."""
    from oracle import oracle as O
    if x is None:
        x = c2_input(shape)
    O.fft3d(np.zeros((4, 4, 4), dtype=np.complex128))  # load + warm caches
    t0 = time.perf_counter()
    y = None
    for _ in range(reps):
        y = O.fft3d(x, threads=threads)
        O.fft3d(y, inverse=True, threads=threads)
    dt = time.perf_counter() - t0
    return reps * 2 * flops_per_transform(shape) / dt / 1e9, dt, y


def port_calibration():
    """The oracle port on ONE host thread against the reference's published
    single-thread forward latencies (same lengths and precisions).  factor =
    port time / published time; > 1 means the port is slower than the
    reference, so CPU ratios against the port overstate the GPU's lead by
    about that factor.  Bounded: well under a second of CPU work."""
    from oracle import oracle as O
    rows = []
    for (prec, n), pub_ns in sorted(PUBLISHED_NS.items()):
        dt = np.complex128 if prec == "f64" else np.complex64
        lanes = max(1, min(2048, (1 << 18) // n))
        rng = np.random.default_rng(n)
        x = (rng.uniform(-1, 1, (lanes, n)) + 1j * rng.uniform(-1, 1, (lanes, n))).astype(dt)
        O.fft1d(x[:1], threads=1)
        best = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            O.fft1d(x, threads=1)
            best = min(best, (time.perf_counter() - t0) / lanes)
        rows.append({"precision": prec, "n": n, "port_ns": round(best * 1e9, 1), "published_ns": pub_ns,
                     "factor": round(best * 1e9 / pub_ns, 3)})
    gm = float(np.exp(np.mean([np.log(r["factor"]) for r in rows])))
    return {"factor_geomean": round(gm, 3), "rows": rows,
            "note": "oracle port, one thread, per-transform time over a batch of lanes; published = reference "
                    "benchmark_results.md (criterion, clone-inclusive) and checklist.md dev-log N=4096"}


def run_reference(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = O.max_threads()
    x = c2_input(SHAPE)
    vals = []
    for _ in range(args.warmup):
        cpu_transform_gflops(SHAPE, 1, x=x)
    for _ in range(args.steps):
        g, _, _ = cpu_transform_gflops(SHAPE, 1, x=x)
        vals.append(g)
    v = float(np.mean(vals))
    step_s = 2 * flops_per_transform(SHAPE) / (v * 1e9)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_s * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1) re/im)",
        "config": c2_config(SHAPE, "f64", args.gpus),
        "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": threads, "kind": "port",
                         "sample": "one forward+inverse of the 256^3 complex128 volume per step (oracle FftPlan3D<f64>)"},
        "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "port_calibration": port_calibration(),
    }
    print(json.dumps(line), flush=True)
    return 0


def time_device(plan, x, y, steps, warmup, torch):
    """fwd (x->y) + inv (y->x) per step; returns seconds per step (CUDA events)."""
    for _ in range(warmup):
        plan.execute(x, out=y)
        plan.execute(y, out=x, inverse=True)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        plan.execute(x, out=y)
        plan.execute(y, out=x, inverse=True)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def link_bandwidth(torch, nbytes, dev):
    """Pinned host <-> device copy bandwidth (GB/s) of one nbytes copy each way."""
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = {}
    for name, fn in (("h2d_gbs", lambda: d.copy_(h, non_blocking=True)),
                     ("d2h_gbs", lambda: h.copy_(d, non_blocking=True))):
        fn()
        torch.cuda.synchronize()
        t = _events_time(fn, 3, 1, torch)
        out[name] = round(nbytes / t / 1e9, 1)
    del h, d
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--shape", default=None, help="override the 3D shape, e.g. 128,256,256 (profiling cases)")
    ap.add_argument("--precision", default=None, choices=["f64", "f32", "tc_bf16", "tc_fp16"])
    ap.add_argument("--profile-case", default=None, choices=["c1", "c2", "c3", "c4", "c5"],
                    help="run one small case of a configuration --reps times and exit (for profiler captures)")
    ap.add_argument("--reps", type=int, default=1, help="--profile-case: repetitions")
    ap.add_argument("--rows", type=int, default=8192, help="--profile-case c4: rows of 4096")
    ap.add_argument("--mode", type=int, default=2, help="--profile-case c3: batch mode")
    ap.add_argument("--c3-class", default="all",
                    choices=["all", "pow2", "smooth", "primes_lt1024", "primes_1024_8191", "primes_ge8192"],
                    help="--profile-case c3: one length class of the batch")
    ap.add_argument("--batch", type=int, default=2, help="--profile-case c5: images of 2048^2")
    ap.add_argument("--quick", action="store_true", help="headline only: no other configurations, e2e or CPU legs")
    ap.add_argument("--workload", default="c2",
                    choices=["c1", "c2", "c3", "c4", "c5", "calib", "stft", "czt", "nufft", "nufft3d", "hilbert"],
                    help="c2 (default) is the headline; the others print their own lines")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.precision is None:
        args.precision = "f64"
    if args.precision not in ("f64", "f32"):
        ap.error("the headline runs f64 or f32")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "calib":
        print(json.dumps({"workload": "calib", "port_calibration": port_calibration()}), flush=True)
        return 0
    if args.workload != "c2":
        return run_secondary(args)

    import torch
    import apollofft_b200 as afc

    global SHAPE
    if args.shape:
        SHAPE = tuple(int(v) for v in args.shape.split(","))
    prec = args.precision
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    hbm_peak, peak_kind = load_peaks()

    x_host = c2_input(SHAPE, seed=2 + rank)
    x = torch.from_numpy(x_host).to(dev, cdt)
    x0 = x.clone()
    y = torch.empty_like(x)
    plan = afc.CudaPlan(list(SHAPE), precision=prec, device=local)

    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            plan.execute(x, out=y)
            plan.execute(y, out=x, inverse=True)
        torch.cuda.synchronize()
        barrier(world)
        n1 = afc.kernel_launch_count()
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.start()
        e0.record(st)
        for _ in range(args.steps):
            plan.execute(x, out=y)
            plan.execute(y, out=x, inverse=True)
        e1.record(st)
        torch.cuda.synchronize()
        clk.stop()
        t_step = e0.elapsed_time(e1) / 1e3 / args.steps
        n2 = afc.kernel_launch_count()
    t_step_max = max_over_ranks(t_step, world, dev)
    launches = n2 - n1
    launches_per_step = launches / args.steps
    roundtrip_err = (torch.linalg.vector_norm(x - x0) / torch.linalg.vector_norm(x0)).item()
    del x0

    flops_step = 2 * flops_per_transform(SHAPE)
    value = world * flops_step / t_step_max / 1e9
    vol_bytes = bytes_per_transform(SHAPE, prec)  # algorithmic: read + write of the volume, per transform
    achieved = 2 * vol_bytes / t_step / 1e9     # = per launch: the transform's bytes over its launches
    per_pass = vol_bytes / (t_step / launches_per_step) / 1e9  # one launch's own read + write of the volume

    # error of the headline forward against the oracle (rank 0): same host input
    err_oracle = None
    cpu = None
    ref_fwd = None
    if rank == 0 and world == 1 and not args.no_cpu and not args.quick and prec == "f64":
        from oracle import oracle as O
        gcpu, _, ref_fwd = cpu_transform_gflops(SHAPE, 1, x=x_host)
        cpu = {"value": round(gcpu, 3), "unit": "GFLOP/s", "cores": O.max_threads(), "kind": "port",
               "sample": "one forward+inverse of the 256^3 complex128 volume (oracle FftPlan3D<f64>, all threads)"}
        yt = plan.execute(torch.from_numpy(x_host).to(dev)).cpu().numpy()
        err_oracle = float(np.linalg.norm(yt - ref_fwd) / np.linalg.norm(ref_fwd))
        del yt

    # other shapes / dtypes of the configuration, each against the oracle
    also = []
    del y
    with_oracle = rank == 0 and world == 1 and not args.no_cpu
    for shp, pa_prec in ([] if args.quick else ALSO):
        dt = torch.complex128 if pa_prec == "f64" else torch.complex64
        xh = c2_input(shp, seed=2)
        xa = torch.from_numpy(xh).to(dev, dt)
        ya = torch.empty_like(xa)
        pa = afc.CudaPlan(list(shp), precision=pa_prec, device=local)
        ts = time_device(pa, xa, ya, max(3, args.steps // 2), args.warmup, torch)
        err = None
        if with_oracle:
            from oracle import oracle as O
            ref = ref_fwd if (shp == SHAPE and ref_fwd is not None) else O.fft3d(xh)
            out = pa.execute(torch.from_numpy(xh).to(dev, dt)).cpu().numpy()
            err = float(np.linalg.norm(out - ref) / np.linalg.norm(ref))
            del out, ref
        also.append({"config": "C2", "shape": list(shp), "precision": pa_prec, "ms_per_step": round(ts * 1e3, 4),
                     "gflops": round(2 * flops_per_transform(shp) / ts / 1e9, 2),
                     "hbm_frac": round((2 * bytes_per_transform(shp, pa_prec) / ts / 1e9) / hbm_peak, 4),
                     "rel_l2_vs_oracle": err})
        del xa, ya, pa
        torch.cuda.empty_cache()
    if not args.quick:
        steps2 = max(3, args.steps // 2)
        for fn in (c1_entry, c3_entry, c4_entry, c5_entry):
            also.append(fn(afc, torch, dev, steps2, args.warmup, hbm_peak, with_oracle))
            torch.cuda.empty_cache()

    # end to end through the host-pointer C-ABI call, pinned buffers
    hx = torch.from_numpy(x_host.astype(np.complex128 if prec == "f64" else np.complex64)).pin_memory()
    hy = torch.empty_like(hx).pin_memory()
    hz = torch.empty_like(hx).pin_memory()
    xn, yn, zn = hx.numpy(), hy.numpy(), hz.numpy()
    L = afc._lib.lib()
    for _ in range(2):
        afc._lib.check(L.afc_execute_host(plan._h, xn.ctypes.data, yn.ctypes.data, 0))
        afc._lib.check(L.afc_execute_host(plan._h, yn.ctypes.data, zn.ctypes.data, 1))
    e2e_steps = 0 if args.quick else max(3, args.steps // 4)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        afc._lib.check(L.afc_execute_host(plan._h, xn.ctypes.data, yn.ctypes.data, 0))
        afc._lib.check(L.afc_execute_host(plan._h, yn.ctypes.data, zn.ctypes.data, 1))
    t_e2e = (time.perf_counter() - t0) / max(e2e_steps, 1)
    t_e2e = max_over_ranks(t_e2e, world, dev)
    e2e_val = world * flops_step / t_e2e / 1e9
    link = None if args.quick else link_bandwidth(torch, int(vol_bytes // 2), dev)
    del hx, hy, hz

    if rank == 0:
        io_bytes = int(2 * (16 if prec == "f64" else 8) * np.prod(SHAPE))
        e2e = None
        if not args.quick:
            # each afc_execute_host call copies the volume in and out, serialized
            bound_s = (io_bytes / 2) / (link["h2d_gbs"] * 1e9) + (io_bytes / 2) / (link["d2h_gbs"] * 1e9)
            e2e = {"value": round(e2e_val, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": io_bytes,
                   "d2h_bytes_per_step": io_bytes, "link": link,
                   "copy_bound_gflops": round(flops_step / (2 * bound_s) / 1e9, 1)}
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_step_max * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": prec, "data": "synthetic (seeded N(0,1) re/im)",
            "config": c2_config(SHAPE, prec, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(achieved / hbm_peak, 4), "traffic": None,
                         "traffic_source": "DRAM bytes per launch: ncu capture summarized in profiles/ "
                                           "(not measured inside this run)",
                         "kernel": f"all launches of the step ({launches_per_step:.0f} per step)",
                         "bytes_definition": "2 N sizeof(complex) per transform, intermediate passes not counted",
                         "per_pass_frac": round(per_pass / hbm_peak, 4),
                         "peak_source": peak_kind},
            "error_vs_oracle_rel_l2": err_oracle,
            "roundtrip_rel_l2": roundtrip_err,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "also": also,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def profile_case(a):
    """One small single-GPU case of a measured configuration, run --reps times
    on seeded device data (inputs larger than the 126 MB L2 where the workload
    allows), for profiler captures, e.g.

        ncu --set full --clock-control none -k regex:tc_fft_kernel -c 1 -o prof \
            python bench.py --profile-case c4 --rows 8192 --precision tc_fp16

    c1  64 x 4096 complex128 forward + inverse
    c2  3D C2C forward + inverse of --shape (default 128,256,256) at --precision f64|f32
    c3  the 4096-length uneven complex64 batch, --mode 0 (graph) | 1 (per length) | 2 (persistent),
        --c3-class one length class of it
    c4  --rows x 4096 complex64 forward at --precision f32 | tc_bf16 | tc_fp16
    c5  --batch x 2048 x 2048 real f32 R2C (full spectrum) forward + adjoint
    """
    import torch
    import apollofft_b200 as afc
    from apollofft_b200 import workloads as W

    g = torch.Generator(device="cuda").manual_seed(7)
    if a.profile_case == "c1":
        x = torch.from_numpy(W.c1_input()).cuda()
        p = afc.CudaPlan([4096], precision="f64", batch=64)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
            p.execute(y, out=x, inverse=True)
    elif a.profile_case == "c2":
        prec = a.precision or "f64"
        shape = [int(v) for v in (a.shape or "128,256,256").split(",")]
        dt = torch.complex128 if prec == "f64" else torch.complex64
        x = torch.randn(shape, dtype=dt, device="cuda", generator=g)
        p = afc.CudaPlan(shape, precision=prec)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
            p.execute(y, out=x, inverse=True)
    elif a.profile_case == "c3":
        lens = W.c3_lengths()
        if a.c3_class != "all":
            def prime(v):
                v = int(v)
                return v > 1 and all(v % d for d in range(2, int(v ** 0.5) + 1))
            keep = {"pow2": lambda v: v & (v - 1) == 0,
                    "smooth": lambda v: v & (v - 1) != 0 and not prime(v),
                    "primes_lt1024": lambda v: prime(v) and v < 1024,
                    "primes_1024_8191": lambda v: prime(v) and 1024 <= v < 8192,
                    "primes_ge8192": lambda v: prime(v) and v >= 8192}[a.c3_class]
            lens = np.asarray([v for v in lens if keep(int(v))], dtype=np.int64)
        x = torch.from_numpy(W.c3_values(lens)).cuda()
        bp = afc.BatchPlan(lens, precision="f32")
        y = torch.empty_like(x)
        for _ in range(a.reps):
            bp.execute(x, out=y, mode=a.mode)
    elif a.profile_case == "c4":
        prec = a.precision or "f32"
        x = torch.randn(a.rows, 4096, dtype=torch.complex64, device="cuda", generator=g)
        p = afc.CudaPlan([4096], precision=prec, batch=a.rows)
        y = torch.empty_like(x)
        for _ in range(a.reps):
            p.execute(x, out=y)
    else:
        from apollofft_b200 import autograd as AG
        img = torch.randn(a.batch, 2048, 2048, dtype=torch.float32, device="cuda", generator=g, requires_grad=True)
        for _ in range(a.reps):
            X = AG.rfft2(img, half=False)
            (X.abs() ** 2).sum().backward()
    torch.cuda.synchronize()
    print("ok")
    return 0


def _events_time(fn, steps, warmup, torch):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def c1_entry(afc, torch, dev, steps, warmup, hbm_peak, with_oracle):
    """C1: 64 x 4096 complex128, forward + inverse per step (U[-1, 1), seed 1)."""
    from apollofft_b200 import workloads as W
    xin = W.c1_input()
    x = torch.from_numpy(xin).to(dev)
    y = torch.empty_like(x)
    p = afc.CudaPlan([4096], precision="f64", batch=64)
    t = _events_time(lambda: (p.execute(x, out=y), p.execute(y, out=x, inverse=True)), steps, warmup, torch)
    fl = 2 * 64 * 5 * 4096 * 12
    out = {"config": "C1", "workload": "1D C2C f64 N=4096 x64 fwd+inv", "us_per_step": round(t * 1e6, 2),
           "gflops": round(fl / t / 1e9, 2), "hbm_frac": round(2 * 2 * 64 * 4096 * 16 / t / 1e9 / hbm_peak, 4)}
    # the same two calls replayed from a CUDA graph: device time without per-call host work
    try:
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(3):
                p.execute(x, out=y)
                p.execute(y, out=x, inverse=True)
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            p.execute(x, out=y)
            p.execute(y, out=x, inverse=True)
        tg = _events_time(g.replay, steps, warmup, torch)
        out["graph_us_per_step"] = round(tg * 1e6, 2)
        out["graph_hbm_frac"] = round(2 * 2 * 64 * 4096 * 16 / tg / 1e9 / hbm_peak, 4)
        del g
    except Exception as exc:  # capture refused: report the host-driven figure only
        out["graph_us_per_step"] = None
        out["graph_error"] = str(exc)[:200]
    if with_oracle:
        from oracle import oracle as O
        ref = O.fft1d(xin)
        got = p.execute(torch.from_numpy(xin).to(dev)).cpu().numpy()
        out["rel_l2_vs_oracle"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return out


def c3_entry(afc, torch, dev, steps, warmup, hbm_peak, with_oracle):
    """C3: 4096 uneven complex64 lengths in one persistent launch per phase (CUDA graph)."""
    from apollofft_b200 import workloads as W
    lens = W.c3_lengths()
    xv = W.c3_values(lens)
    x = torch.from_numpy(xv).to(dev)
    t0 = time.perf_counter()
    bp = afc.BatchPlan(lens, precision="f32")
    plan_s = time.perf_counter() - t0
    y = torch.empty_like(x)
    fl = float(np.sum(5.0 * lens * np.log2(lens)))
    by = float(np.sum(2.0 * lens * 8))
    t = _events_time(lambda: bp.execute(x, out=y, mode=0), steps, warmup, torch)
    tp = _events_time(lambda: bp.execute(x, out=y, mode=1), 2, 1, torch)
    out = {"config": "C3", "workload": "4096 uneven 1D complex64 lengths log-uniform [64, 65536], thirds "
                                       "pow2/7-smooth/prime, forward", "us": round(t * 1e6, 1),
           "gflops": round(fl / t / 1e9, 1), "hbm_frac": round(by / t / 1e9 / hbm_peak, 4),
           "per_size_launches_us": round(tp * 1e6, 1), "plan_seconds": round(plan_s, 2)}
    if with_oracle:
        from oracle import oracle as O
        yy = bp.execute(x, mode=0).cpu().numpy()
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
        sel = np.arange(0, len(lens), 16)
        sx = np.concatenate([xv[offs[i]:offs[i] + lens[i]] for i in sel]).astype(np.complex128)
        so = np.concatenate([[0], np.cumsum(lens[sel])[:-1]])
        ref = O.fft_uneven(sx, so, lens[sel])
        errs, defects = [], []
        for i, o in zip(sel, so):
            r = ref[o:o + lens[i]]
            exact = np.fft.fft(sx[o:o + lens[i]])
            # the reference's Rader for some primes (10831, 16811) recurses into a
            # prime power its dispatcher leaves untransformed: not a DFT there
            if np.linalg.norm(r - exact) > 1e-10 * np.linalg.norm(exact):
                defects.append(int(lens[i]))
                r = exact
            errs.append(np.linalg.norm(yy[offs[i]:offs[i] + lens[i]] - r) / np.linalg.norm(r))
        out["rel_l2_vs_oracle_max_sampled_lanes"] = float(max(errs))
        out["oracle_sample"] = f"every 16th lane ({len(sel)} lanes), f64 oracle per-length dispatch"
        out["reference_defect_lanes_vs_exact_dft"] = defects
    return out


def c4_entry(afc, torch, dev, steps, warmup, hbm_peak, with_oracle):
    """C4: 16384 x 4096 complex64 forward; FP32 SIMT vs the split-precision tensor-core forms."""
    from apollofft_b200 import workloads as W
    xs, k = W.c4_rows()
    x = torch.from_numpy(xs).to(dev)
    fl = 16384 * 5 * 4096 * 12
    ref = None
    if with_oracle:
        from oracle import oracle as O
        ref = O.fft1d(xs.astype(np.complex128))
        den = np.linalg.norm(ref, axis=1)
    variants = {}
    t32 = None
    for name, prec in (("fp32_simt", "f32"), ("tc_bf16_split", "tc_bf16"), ("tc_fp16_split", "tc_fp16")):
        p = afc.CudaPlan([4096], precision=prec, batch=16384)
        y = torch.empty_like(x)
        t = _events_time(lambda: p.execute(x, out=y), steps, warmup, torch)
        v = {"us": round(t * 1e6, 1), "gflops": round(fl / t / 1e9, 1),
             "hbm_frac": round(2 * 16384 * 4096 * 8 / t / 1e9 / hbm_peak, 4)}
        if t32 is None:
            t32 = t
        else:
            v["speedup_vs_fp32_simt"] = round(t32 / t, 3)
        if ref is not None:
            yc = y.cpu().numpy()
            r = np.linalg.norm(yc - ref, axis=1) / den
            v["rel_l2_per_row_max_vs_oracle"] = float(r.max())
            v["rel_l2_per_row_median_vs_oracle"] = float(np.median(r))
            v["rel_l2_per_row_max_hdr_rows"] = float(r[k != 0].max())
        variants[name] = v
        del p, y
    return {"config": "C4", "workload": "16384 x 4096 complex64 forward, 25% rows x 10^k (k in [-6, 6])",
            "variants": variants}


def c5_entry(afc, torch, dev, steps, warmup, hbm_peak, with_oracle):
    """C5: 8 x 2048^2 real f32, full-spectrum R2C, loss sum |w X|^2, gradient by the adjoint."""
    from apollofft_b200 import autograd as AG
    from apollofft_b200 import workloads as W
    rng = np.random.default_rng(5)
    img_h = rng.standard_normal((8, 2048, 2048)).astype(np.float32)
    img = torch.from_numpy(img_h).to(dev)
    w = torch.from_numpy(W.radial_weight(2048)).to(dev).to(torch.float32)

    def fwd():
        with torch.no_grad():
            return torch.sum(torch.abs(w * AG.rfft2(img)) ** 2)

    xg = img.clone().requires_grad_(True)

    def fwdbwd():
        xg.grad = None
        loss = torch.sum(torch.abs(w * AG.rfft2(xg)) ** 2)
        loss.backward()

    p = afc.CudaPlan([2048, 2048], precision="f32", kind="r2c_full", batch=8)
    yb = torch.empty((8, 2048, 2048), dtype=torch.complex64, device=dev)
    tr = _events_time(lambda: p.execute(img, out=yb), steps, warmup, torch)
    tf = _events_time(fwd, steps, warmup, torch)
    tb = _events_time(fwdbwd, steps, warmup, torch)
    N = 2048 * 2048
    fl = 8 * 2.5 * N * math.log2(N)
    r2c_bytes = 8 * N * (4 + 8)  # real input + full complex spectrum
    out = {"config": "C5", "workload": "8 x 2048^2 f32 real, full-spectrum R2C (reference contract), loss sum |w X|^2",
           "r2c_forward_ms": round(tr * 1e3, 3), "r2c_gflops": round(fl / tr / 1e9, 1),
           "r2c_hbm_frac": round(r2c_bytes / tr / 1e9 / hbm_peak, 4),
           "loss_forward_ms": round(tf * 1e3, 3), "loss_forward_backward_ms": round(tb * 1e3, 3),
           "backward_over_forward": round(tb / tf, 3)}
    if with_oracle:
        from oracle import oracle as O
        ref = O.fft2d(img_h.astype(np.complex128))
        got = yb.cpu().numpy()
        out["rel_l2_vs_oracle"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    del xg, img, yb
    return out


def run_secondary(args):
    """Lines for the other configurations (not the headline)."""
    import torch
    import apollofft_b200 as afc
    from apollofft_b200 import workloads as W
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    hbm_peak, peak_kind = load_peaks()
    line = {"workload": args.workload, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "peak_gbs": hbm_peak}
    if args.workload in ("c1", "c3", "c4", "c5"):
        fn = {"c1": c1_entry, "c3": c3_entry, "c4": c4_entry, "c5": c5_entry}[args.workload]
        line.update(fn(afc, torch, dev, args.steps, args.warmup, hbm_peak, True))
        from oracle import oracle as O
        if args.workload == "c1":
            xin = W.c1_input()
            fl = 2 * 64 * 5 * 4096 * 12
            t0 = time.perf_counter()
            reps = 20
            for _ in range(reps):
                O.fft1d(O.fft1d(xin), inverse=True)
            tc = (time.perf_counter() - t0) / reps
            line["cpu_baseline"] = {"value": round(fl / tc / 1e9, 2), "unit": "GFLOP/s", "cores": O.max_threads(),
                                    "kind": "port", "sample": f"{reps} x (64 x 4096 fwd+inv)"}
        elif args.workload == "c3":
            lens = W.c3_lengths()
            xv = W.c3_values(lens)
            offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
            sample = slice(0, len(lens), 16)
            sl = lens[sample]
            so = np.concatenate([[0], np.cumsum(sl)[:-1]])
            sx = np.concatenate([xv[o:o + n] for o, n in zip(offs[sample], sl)])
            t0 = time.perf_counter()
            O.fft_uneven(sx, so, sl)
            tc = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(float(np.sum(5.0 * sl * np.log2(sl))) / tc / 1e9, 3),
                                    "unit": "GFLOP/s", "cores": O.max_threads(), "kind": "port",
                                    "sample": f"every 16th lane ({len(sl)} lanes), oracle per-length dispatch f32"}
    elif args.workload == "stft":
        # apollo-stft's analysis loop (frame copy + window + one FFT per frame) fused
        # into the FFT load: 2^22 f64 samples, frame 1024, hop 256 (seeded N(0,1))
        from apollofft_b200.stft import StftPlan
        n_sig, frame_len, hop = 1 << 22, 1024, 256
        sig_np = np.random.default_rng(11).standard_normal(n_sig)
        sig = torch.from_numpy(sig_np).to(dev)
        plan = StftPlan(frame_len, hop, precision="f64")
        frames = plan.frame_count(n_sig)
        out = torch.empty((frames, frame_len), dtype=torch.complex128, device=dev)
        t = _events_time(lambda: plan.forward(sig, out=out), args.steps, args.warmup, torch)
        fl = frames * 5 * frame_len * math.log2(frame_len)
        byts = n_sig * 8 + frames * frame_len * 16
        line.update({"metric": "GFLOP/s", "value": round(fl / t / 1e9, 1), "ms_per_step": round(t * 1e3, 4),
                     "frames_per_s": round(frames / t, 1), "hbm_frac": round(byts / t / 1e9 / hbm_peak, 4),
                     "config": f"STFT analysis f64: {n_sig} samples, frame {frame_len}, hop {hop}, {frames} frames, "
                               "Hann window, one fused launch"})
        # the reference's pattern on the host: per frame, window into a slice and
        # transform it (oracle FftPlan1D<f64>), frames over all threads; bounded sample
        from oracle import oracle as O
        sub = min(frames, 4096)
        win = plan.window
        fr = np.zeros((sub, frame_len), dtype=np.complex128)
        for m in range(sub):
            st0 = m * hop - frame_len // 2
            lo, hi = max(st0, 0), min(st0 + frame_len, n_sig)
            fr[m, lo - st0:hi - st0] = sig_np[lo:hi] * win[lo - st0:hi - st0]
        t0 = time.perf_counter()
        ref = O.fft1d(fr)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(sub * 5 * frame_len * math.log2(frame_len) / tc / 1e9, 2),
                                "unit": "GFLOP/s", "cores": O.max_threads(), "kind": "port",
                                "sample": f"first {sub} frames: window + oracle FFT per frame (frame gather not timed)"}
        got = out[:sub].cpu().numpy()
        line["error_vs_oracle_rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    elif args.workload == "czt":
        # apollo-czt's Bluestein path (premultiply, two FFTs, kernel product,
        # postmultiply) as one launch: 4096 lanes, n = m = 1000, zoom on an arc (f64)
        import cmath
        from apollofft_b200.czt import CztPlan
        lanes, n, m = 4096, 1000, 1000
        a, w = cmath.exp(0.3j), cmath.exp(-2j * cmath.pi / 4000)
        rng = np.random.default_rng(12)
        xn = rng.uniform(-1, 1, (lanes, n)) + 1j * rng.uniform(-1, 1, (lanes, n))
        x = torch.from_numpy(xn).to(dev)
        plan = CztPlan(n, m, a, w, precision="f64")
        out = torch.empty((lanes, m), dtype=torch.complex128, device=dev)
        t = _events_time(lambda: plan.forward(x, out=out), args.steps, args.warmup, torch)
        Lc = plan.convolution_len()
        fl = lanes * 2 * 5 * Lc * math.log2(Lc)  # two length-L FFTs per lane
        line.update({"metric": "GFLOP/s", "value": round(fl / t / 1e9, 1), "ms_per_step": round(t * 1e3, 4),
                     "transforms_per_s": round(lanes / t, 1),
                     "hbm_frac": round(lanes * (n + m) * 16 / t / 1e9 / hbm_peak, 4),
                     "config": f"CZT f64: {lanes} lanes, n = m = {n}, convolution {Lc}, A = e^0.3i, W = e^(-2 pi i/4000)"})
        from oracle import oracle as O
        cn = np.array([cmath.rect(abs(a) ** -j, cmath.phase(a) * -j) * cmath.rect(1.0, cmath.phase(w) * 0.5 * j * j)
                       for j in range(n)])
        ck = np.array([cmath.rect(1.0, cmath.phase(w) * 0.5 * k * k) for k in range(m)])
        ker = np.zeros(Lc, dtype=np.complex128)
        for k in range(m):
            ker[k] = cmath.rect(1.0, -cmath.phase(w) * 0.5 * k * k)
        for j in range(1, n):
            ker[Lc - j] = cmath.rect(1.0, -cmath.phase(w) * 0.5 * j * j)
        sub = 512
        t0 = time.perf_counter()
        fk = O.fft1d(ker)
        ws = np.zeros((sub, Lc), dtype=np.complex128)
        ws[:, :n] = xn[:sub] * cn
        ws = O.fft1d(O.fft1d(ws) * fk, inverse=True)
        ref = ws[:, :m] * ck
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(sub * 2 * 5 * Lc * math.log2(Lc) / tc / 1e9, 2), "unit": "GFLOP/s",
                                "cores": O.max_threads(), "kind": "port",
                                "sample": f"{sub} lanes: premultiply, oracle FFTs, product, postmultiply"}
        line["error_vs_reference_path_rel_l2"] = float(np.linalg.norm(out[:sub].cpu().numpy() - ref) / np.linalg.norm(ref))
    elif args.workload == "nufft":
        # apollo-nufft NufftPlan1D at the reference defaults (sigma 2, width 6):
        # n = 65536 bins, 2^20 uniform random points; type 1 then type 2 per step (f64)
        from apollofft_b200.nufft import NufftPlan1D
        n, npts, dx = 65536, 1 << 20, 1.0 / 65536
        rng = np.random.default_rng(13)
        pos_np = rng.uniform(0.0, 1.0, npts)
        val_np = rng.standard_normal(npts) + 1j * rng.standard_normal(npts)
        pos = torch.from_numpy(pos_np).to(dev)
        val = torch.from_numpy(val_np).to(dev)
        plan = NufftPlan1D(n, dx)
        f = torch.empty(n, dtype=torch.complex128, device=dev)
        back = torch.empty(npts, dtype=torch.complex128, device=dev)
        t = _events_time(lambda: (plan.type1(pos, val, out=f), plan.type2(f, pos, out=back)), args.steps,
                         args.warmup, torch)
        line.update({"metric": "points/s", "value": round(2 * npts / t, 1), "ms_per_step": round(t * 1e3, 4),
                     "config": f"NUFFT 1D f64 type 1 + type 2: n = {n}, {npts} points, sigma 2, kernel width 6"})
        # error of type 1 against the exact sum on 64 sampled bins
        ks = np.array([k if k <= n // 2 else k - n for k in range(0, n, n // 64)])
        exact = np.exp(-2j * np.pi * np.outer(ks, pos_np)) @ val_np
        got = f.cpu().numpy()[np.arange(0, n, n // 64)]
        line["type1_rel_l2_vs_exact_sampled_bins"] = float(np.linalg.norm(got - exact) / np.linalg.norm(exact))
        # the reference's plan restated in C++ (oracle/nufft_oracle.cpp), one thread as
        # the reference runs it, on the same points
        from oracle import nufft as ON
        t0 = time.perf_counter()
        fr = ON.c_type1_1d(n, dx, 2, 6, pos_np, val_np)
        ON.c_type2_1d(n, dx, 2, 6, fr, pos_np)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(2 * npts / tc, 1), "unit": "points/s", "cores": 1, "kind": "port",
                                "sample": f"type 1 + type 2 of all {npts} points, same plan (C++ restatement, "
                                "one thread)"}
    elif args.workload == "hilbert":
        # apollo-hilbert's analytic_signal_into (forward, mask, normalized inverse)
        # as one fused launch: 4096 lanes of 4096 f64 samples (seeded N(0,1))
        from apollofft_b200.hilbert import HilbertPlan
        lanes, n = 4096, 4096
        xn = np.random.default_rng(16).standard_normal((lanes, n))
        x = torch.from_numpy(xn).to(dev)
        plan = HilbertPlan(n)
        out = torch.empty((lanes, n), dtype=torch.complex128, device=dev)
        t = _events_time(lambda: plan.analytic_signal(x, out=out), args.steps, args.warmup, torch)
        fl = lanes * 2 * 5 * n * math.log2(n)  # two length-n transforms per lane
        byts = lanes * n * (8 + 16)
        line.update({"metric": "GFLOP/s", "value": round(fl / t / 1e9, 1), "ms_per_step": round(t * 1e3, 4),
                     "signals_per_s": round(lanes / t, 1), "hbm_frac": round(byts / t / 1e9 / hbm_peak, 4),
                     "config": f"analytic signal f64: {lanes} lanes x {n}, one fused launch"})
        from oracle import oracle as O
        sub = 512
        k = np.arange(n)
        mask = np.where(k < (n + 1) // 2, 2.0, 0.0)
        mask[0] = 1.0
        mask[n // 2] = 1.0
        t0 = time.perf_counter()
        ref = O.fft1d(O.fft1d(xn[:sub].astype(np.complex128)) * mask, inverse=True)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(sub * 2 * 5 * n * math.log2(n) / tc / 1e9, 2), "unit": "GFLOP/s",
                                "cores": O.max_threads(), "kind": "port",
                                "sample": f"{sub} lanes: oracle forward, mask, oracle inverse"}
        line["quadrature_rel_l2_vs_reference_path"] = float(
            np.linalg.norm(out[:sub].cpu().numpy().imag - ref.imag) / np.linalg.norm(ref.imag))
    elif args.workload == "nufft3d":
        # apollo-nufft NufftPlan3D at the reference defaults (sigma 2, width 6):
        # 64^3 modes on the unit cube (oversampled 128^3), 2^18 uniform random
        # points; type 1 then type 2 per step (f64)
        from apollofft_b200.nufft import NufftPlan3D
        nb, npts = 64, 1 << 18
        rng = np.random.default_rng(14)
        pos_np = rng.uniform(0.0, 1.0, (npts, 3))
        val_np = rng.standard_normal(npts) + 1j * rng.standard_normal(npts)
        pos = torch.from_numpy(pos_np).to(dev)
        val = torch.from_numpy(val_np).to(dev)
        plan = NufftPlan3D((nb, nb, nb), (1.0 / nb,) * 3)
        f = torch.empty((nb, nb, nb), dtype=torch.complex128, device=dev)
        back = torch.empty(npts, dtype=torch.complex128, device=dev)
        t1 = _events_time(lambda: plan.type1(pos, val, out=f), args.steps, args.warmup, torch)
        t2 = _events_time(lambda: plan.type2(f, pos, out=back), args.steps, args.warmup, torch)
        t = t1 + t2
        line.update({"metric": "points/s", "value": round(2 * npts / t, 1), "ms_per_step": round(t * 1e3, 4),
                     "type1_ms": round(t1 * 1e3, 4), "type2_ms": round(t2 * 1e3, 4),
                     "config": f"NUFFT 3D f64 type 1 + type 2: {nb}^3 modes, grid {plan.oversampled}, {npts} points, "
                               "sigma 2, kernel width 6"})
        # error of type 1 against the exact sum on 64 sampled modes
        rs = np.random.default_rng(15)
        idx = rs.integers(0, nb, (64, 3))
        ks = np.where(idx <= nb // 2, idx, idx - nb)
        exact = np.exp(-2j * np.pi * ks @ pos_np.T) @ val_np
        fc = f.cpu().numpy()
        got = fc[idx[:, 0], idx[:, 1], idx[:, 2]]
        line["type1_rel_l2_vs_exact_sampled_modes"] = float(np.linalg.norm(got - exact) / np.linalg.norm(exact))
        from oracle import nufft as ON
        sub = 1 << 15
        t0 = time.perf_counter()
        fr = ON.c_type1_3d((nb, nb, nb), (1.0 / nb,) * 3, 2, 6, pos_np[:sub], val_np[:sub])
        ON.c_type2_3d((nb, nb, nb), (1.0 / nb,) * 3, 2, 6, fr, pos_np[:sub])
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(2 * sub / tc, 1), "unit": "points/s", "cores": 1, "kind": "port",
                                "sample": f"type 1 + type 2 of the first {sub} points, same plan (C++ "
                                "restatement, one thread, 3D FFT of the 128^3 grid included)"}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
