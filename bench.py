"""Benchmark: GSHT forward+inverse transforms per second at lmax 1024.

Workload (one "step"): a batch of 64 complex fields at lmax = 1024 on the
Gauss-Legendre grid (nTheta = 1025, nPhi = 2048), upper index n = 0,
coefficients complex standard normal with envelope (l+1)^-1.5 from a fixed
seed; one inverse transform (coefficients -> grid) and one forward transform
(grid -> coefficients, into a zeroed output) per field. Inputs live in HBM
when the timed region starts; each step touches ~1.1 GB of coefficients and
~2.2 GB of grid values, far more than the 126 MB L2, so no flush is needed.

    python bench.py [--gpus N --steps K --warmup W] [--precision fp64|bf16x3|ozaki|ozaki4]
    python bench.py --impl reference     # the reference's CPU path (oracle/_ref)

Multi-GPU runs (torchrun, one process per GPU) are independent replicas: each
rank transforms its own 64 fields (weak scaling; the transform has no
exchange step), timed on the device and reduced with MAX over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GSHT fwd+inv/s, lmax 1024: tensor-core vs FP64 GPU at ≤1e-6 and ≤1e-12 err"
UNIT = "fwd+inv/s"
L_MAX = 1024
N_UPPER = 0
FIELDS = 64
ENVELOPE = 1.5
DTYPE = {"fp64": "f64", "bf16x3": "bf16", "ozaki": "int8", "ozaki4": "int8"}
STAGES = ["prep_inverse", "legendre_inverse", "fft_inverse", "fft_forward",
          "prep_forward", "legendre_forward", "accumulate_forward"]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default=None, choices=[None, "fp64", "bf16x3", "ozaki", "ozaki4"])
    p.add_argument("--fields", type=int, default=FIELDS)
    p.add_argument("--lmax", type=int, default=L_MAX)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--trace", action="store_true",
                   help="after timing, run one traced round trip per tensor-core form and "
                        "add the per-role cycle split of its Legendre kernels to the mode line")
    p.add_argument("--no-secondary", action="store_true",
                   help="skip the batch / large / pipeline workloads the default run adds")
    p.add_argument("--workload", default="headline",
                   choices=["headline", "batch", "large", "pipeline"],
                   help="headline: 64 fields at lmax 1024 (the metric); batch: 256 fields of "
                        "uneven lmax in one CUDA graph vs per-field calls; large: one field at "
                        "lmax 2048 (table streaming, GB/s); pipeline: 64 field-product pairs at "
                        "lmax 768")
    return p.parse_args()


def workload(args):
    return {
        "workload": (f"{args.fields} complex fields, lmax {args.lmax} (nTheta {args.lmax + 1}, "
                     f"nPhi {2 * args.lmax}), upper index n={N_UPPER}, envelope (l+1)^-{ENVELOPE}, "
                     "one inverse + one forward transform per field"),
        "lmax": args.lmax,
        "fields_per_gpu": args.fields,
        "upper_index": N_UPPER,
        "l2": "inputs larger than L2 (coefficients + grids >> 126 MB); no flush",
    }


def coefficients(lmax, fields, seed=0, generator=None):
    """Seeded coefficients of the headline workload. ``generator`` is a
    random_coefficients function (the package's, or the oracle's for the
    reference arm, which must not load the CUDA library)."""
    if generator is None:
        import gshtrans_b200 as gsht

        generator = gsht.random_coefficients
    rng = np.random.default_rng(seed)
    return np.stack([generator(rng, lmax, lmax, N_UPPER, False, ENVELOPE)
                     for _ in range(fields)])


def run_config(args):
    """The config dict both arms print (identical for the same arguments)."""
    return workload(args) | {"parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, its maximum and the clock-event (throttle) reasons, sampled
    while the timed region runs: through NVML every 10 ms where the driver's
    library loads (pynvml; the same counters nvidia-smi prints), otherwise by
    running nvidia-smi every 200 ms. The device is found by its PCI bus id
    when one is given (CUDA and NVML may number GPUs differently), else by
    index."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap,power.draw")
    # NVML clock-event reason bits, in the order of FIELDS' reason columns.
    REASON_BITS = (0x8, 0x40, 0x20, 0x4)

    def __init__(self, index: int, bus_id: str | None = None, nvml=None, period_s: float = 0.01):
        self.index = index
        self.bus_id = bus_id
        self.period_s = period_s
        self.samples = []
        self.source = None
        self._nvml = nvml
        self._stop = threading.Event()
        self._t = None
        self._opened = None

    def _open_nvml(self):
        nv = self._nvml
        if nv is None:
            import pynvml as nv
        nv.nvmlInit()
        h = None
        if self.bus_id:
            try:
                h = nv.nvmlDeviceGetHandleByPciBusId(self.bus_id)
            except Exception:
                h = None
        if h is None:
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
        # Every call is tried once here, so that a driver without one of them
        # falls back to nvidia-smi before the timed region starts.
        reasons = None
        for name in ("nvmlDeviceGetCurrentClocksEventReasons",
                     "nvmlDeviceGetCurrentClocksThrottleReasons"):
            fn = getattr(nv, name, None)
            try:
                if fn is not None:
                    int(fn(h))
                    reasons = fn
                    break
            except Exception:
                continue
        if reasons is None:
            raise RuntimeError("NVML reports no clock-event reasons")
        nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        return nv, h, reasons, nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

    def _sample_nvml(self):
        nv, h, reasons, mx = self._opened
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = int(reasons(h))
            self.samples.append([str(sm), str(mx)] +
                                ["Active" if r & bit else "Not Active" for bit in self.REASON_BITS])
        except Exception:
            pass

    def _run(self):
        if self._opened is not None:
            self.source = "nvml"
            while not self._stop.is_set():
                self._sample_nvml()
                self._stop.wait(self.period_s)
            return
        self.source = "nvidia-smi"
        dev = self.bus_id or str(self.index)
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", dev, f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
                elif dev != str(self.index):
                    dev = str(self.index)  # bus id not accepted: by index
                    continue
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        # NVML is opened here, before the timed region, and sampled once at
        # its start and once at its end, so that a short region still has
        # samples from its own span.
        try:
            self._opened = self._open_nvml()
        except Exception:
            self._opened = None
        if self._opened is not None:
            self._sample_nvml()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if self._opened is not None:
            self._sample_nvml()
            try:
                self._opened[0].nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 2 + i and s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


def pci_bus_id(torch, index: int):
    """domain:bus:device.0 of a CUDA device, as NVML and nvidia-smi -i take it."""
    try:
        p = torch.cuda.get_device_properties(index)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except Exception:
        return None


# ---------------------------------------------------------------------------
# Reference arm: the reference's own CPU implementation (oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_run(lmax, steps, warmup, log=None):
    """Times the reference's round trip (InverseTransformation then
    ForwardTransformation per field, OpenMP over fields) on the host cores.
    Each step transforms one field per core."""
    import oracle

    if not oracle.Reference.available():
        return None, "reference build oracle/_ref/libgsht_ref.so is absent"
    cores = cpu_cores()
    ref = oracle.Reference()
    t0 = time.perf_counter()
    g = ref.grid(lmax, N_UPPER, 0, 2)  # NRange = Single: one host table
    build_s = time.perf_counter() - t0
    coefs = coefficients(lmax, cores, seed=1, generator=oracle.random_coefficients)
    for _ in range(warmup):
        g.roundtrip_batch(lmax, N_UPPER, False, coefs, cores)
    t0 = time.perf_counter()
    for _ in range(steps):
        out = g.roundtrip_batch(lmax, N_UPPER, False, coefs, cores)
    dt = time.perf_counter() - t0
    err = float(np.linalg.norm(out - coefs) / np.linalg.norm(coefs))
    # the reference's own transform is serial: one field on one core
    t1 = time.perf_counter()
    g.roundtrip_batch(lmax, N_UPPER, False, coefs[:1], 1)
    single_s = time.perf_counter() - t1
    g.close()
    value = steps * cores / dt
    return {
        "value": value, "unit": UNIT, "cores": cores, "kind": "reference",
        "sample": (f"{steps} step(s) x {cores} complex field(s) (one per core), lmax {lmax}, "
                   f"inverse+forward each, reference GaussLegendreGrid.h compiled in place "
                   f"(FFTWpp/GaussQuad stand-ins); table build {build_s:.1f} s untimed"),
        "seconds": dt, "round_trip_rel_err": err,
        "single_core_value": 1.0 / single_s,
    }, None


def impl_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    res, why = reference_run(args.lmax, args.steps, args.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    line = {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * res["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": run_config(args), "precision": "fp64",
        "fields_per_step": res["cores"],
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample",
                                             "single_core_value")},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "round_trip_rel_err": res["round_trip_rel_err"],
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def reduce_max_ms(ms: float, dist, device) -> float:
    """Slowest rank's device time: the job's time for replicas run in parallel."""
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank: int) -> int:
    """Each rank transforms its own fields (distinct seeded coefficients)."""
    return 1000 + rank


def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s), best of 3."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def measure_mode(gsht, grid, torch, dev, coef, field, back, precision, args, world, dist):
    """Times args.steps round trips in one precision form (CUDA events on the
    current stream, barrier + synchronize on both sides, MAX over ranks)."""
    import ctypes

    L = args.lmax

    # One step: the inverse of the batch, then its forward, which ADDS into
    # back (ForwardTransformation's += semantics). back is zeroed before the
    # first warm-up step only, for the round-trip check; clearing it is not
    # part of a transform and stays out of the timed steps.
    def step():
        grid.inverse_batch(L, N_UPPER, coef, field, precision)
        grid.forward_batch(L, N_UPPER, field, back, precision)

    back.zero_()
    step()
    torch.cuda.synchronize()
    grid.device_status()
    rt_err = float(torch.linalg.norm(back - coef) / torch.linalg.norm(coef))
    for _ in range(args.warmup - 1):
        step()
    lib = gsht.library
    lib.gsht_profile_enable(1)
    launches0 = gsht.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_device()
    with ClockSampler(cur, pci_bus_id(torch, cur)) as clk:
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = gsht.launch_count() - launches0
    ns = len(STAGES)
    stage_ms = (ctypes.c_double * ns)()
    stage_n = (ctypes.c_long * ns)()
    lib.gsht_profile_read(ctypes.cast(stage_ms, ctypes.c_void_p),
                          ctypes.cast(stage_n, ctypes.c_void_p), ns)
    lib.gsht_profile_enable(0)
    grid.device_status()
    if world > 1:
        ms = reduce_max_ms(ms, dist, dev)
    stages = {STAGES[i]: {"ms_per_step": stage_ms[i] / args.steps,
                          "launches_per_step": stage_n[i] / args.steps} for i in range(ns)}
    trace = None
    if getattr(args, "trace", False) and precision != "fp64":
        # Outside the timed region: one round trip through the traced kernel
        # copies; fractions of each role's cycles (summed over CTAs).
        with gsht.TensorCoreTrace() as tr:
            step()
            trace = {}
            for d, name in ((0, "inverse"), (1, "forward")):
                c = tr.read(precision, d)
                trace[name] = {k: round(v, 4) for k, v in c.items() if "frac" in k}
                trace[name]["ctas"] = int(c["ctas"])
                trace[name]["mma_ctas"] = int(c["mma_ctas"])
                if c["mma_ctas"]:
                    trace[name]["mma_cycles_per_issuer"] = c["mma"] / c["mma_ctas"]
        grid.device_status()
    return {"ms": ms, "launches": launches, "stages": stages, "clocks": clk.summary(),
            "round_trip_rel_err": rt_err,
            "legendre_ms": (stage_ms[1] + stage_ms[5]) / args.steps,
            "legendre_launches": int(stage_n[1] + stage_n[5]), "trace": trace}


def legendre_roofline(precision, res, args, peaks):
    """Roofline of the dominant kernel, the per-order Legendre contraction
    (inverse + forward launches). Algorithmic work: 4 flops per (table entry
    x complex field) per direction; for the tensor-core forms the tensor-pipe
    work is that times the split products (6 BF16 MMAs, 28 INT8 MMAs)."""
    L, B = args.lmax, args.fields
    entries = ((L + 1) ** 2 - N_UPPER ** 2) * (L + 1)
    flops_per_dir = 4.0 * B * entries
    t = res["legendre_ms"] * 1e-3 / 2  # per launch (one direction)
    pipe = {"fp64": 1, "bf16x3": 6, "ozaki": 28, "ozaki4": 10}[precision]
    achieved = pipe * flops_per_dir / t / 1e12
    if precision == "fp64":
        peak, src = peaks.get("fp64"), "cuBLAS DGEMM 8192^3 measured in this run"
        unit = "TFLOP/s"
    elif precision == "bf16x3":
        peak, src = peaks.get("bf16"), "MEASURED_PEAKS.json bf16_tflops (burst, of measured)"
        unit = "TFLOP/s"
    else:
        peak, src = peaks.get("int8"), "2 x MEASURED_PEAKS.json bf16_tflops (dense INT8 = 2x BF16 rate)"
        unit = "TOP/s"
    # DRAM bytes (read + write) per launch, mean of the inverse and forward
    # launches: a constant taken from an earlier ncu capture of this shape
    # (lmax 1024, 64 complex fields, n = 0), not a measurement of this run;
    # None for any other shape.
    traffic = None
    if L == L_MAX and B == 64 and N_UPPER == 0:
        traffic = {"fp64": (7.581e9 + 8.784e9) / 2, "bf16x3": (5.319e9 + 5.987e9) / 2,
                   "ozaki": (7.156e9 + 6.883e9) / 2,
                   "ozaki4": (5.118e9 + 4.678e9) / 2}.get(precision)
    return {
        "kernel": {"fp64": "k_legendre_fp64", "bf16x3": "k_legendre_tc (kind::f16)",
                   "ozaki": "k_legendre_oz (kind::i8)",
                   "ozaki4": "k_legendre_oz (kind::i8, 4 slices)"}[precision] + " inverse+forward",
        "bound": "tensor", "achieved": achieved, "peak": peak, "unit": unit,
        "frac": achieved / peak if peak else None, "peak_source": src,
        "algorithmic_flops_per_launch": flops_per_dir,
        "tensor_ops_per_launch": pipe * flops_per_dir,
        "avg_launch_ms": 1e3 * t, "traffic": traffic,
        "traffic_source": ("constant from an earlier ncu capture of this shape "
                           "(dram__bytes_read.sum + dram__bytes_write.sum per launch), "
                           "not measured in this run") if traffic is not None else None,
    }


def impl_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import gshtrans_b200 as gsht

    modes = [args.precision] if args.precision else ["ozaki", "ozaki4", "bf16x3", "fp64"]
    headline = modes[0]
    L, B = args.lmax, args.fields
    grid = gsht.GaussLegendreGrid(L, N_UPPER, nrange=gsht.Single,
                                  forms=[m for m in modes if m != "fp64"])
    coef_h = coefficients(L, B, seed=replica_seed(rank))
    coef = torch.from_numpy(coef_h).to(dev)
    field = torch.empty((B, grid.FieldSize()), dtype=torch.complex128, device=dev)
    back = torch.zeros_like(coef)

    # Each form is timed in its own loop; the GPU idles a few seconds before
    # each, so that every form starts from a similar thermal and power state
    # (a dense tensor-core loop leaves the part near its power cap, which
    # would otherwise slow whichever form runs next).
    results = {}
    for i, m in enumerate(modes):
        if i:
            time.sleep(3.0)
        results[m] = measure_mode(gsht, grid, torch, dev, coef, field, back, m, args, world, dist)
    # accuracy of each form against the FP64 path on the same inputs
    ref_f = ref_c = None
    if "fp64" in modes and len(modes) > 1:
        ref_f = torch.empty_like(field)
        grid.inverse_batch(L, N_UPPER, coef, ref_f, "fp64")
        ref_c = torch.zeros_like(coef)
        grid.forward_batch(L, N_UPPER, ref_f, ref_c, "fp64")
        for m in modes:
            f = torch.empty_like(field)
            grid.inverse_batch(L, N_UPPER, coef, f, m)
            c = torch.zeros_like(coef)
            grid.forward_batch(L, N_UPPER, ref_f, c, m)
            results[m]["inverse_rel_err_vs_fp64"] = float(torch.linalg.norm(f - ref_f) / torch.linalg.norm(ref_f))
            results[m]["forward_rel_err_vs_fp64"] = float(torch.linalg.norm(c - ref_c) / torch.linalg.norm(ref_c))
            del f, c
        del ref_f, ref_c
    torch.cuda.synchronize()
    peaks = {}
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        mpj = json.load(open(mp))
        peaks["bf16"] = mpj.get("bf16_tflops")
        peaks["int8"] = 2 * mpj["bf16_tflops"] if mpj.get("bf16_tflops") else None
    if "fp64" in modes:
        peaks["fp64"] = measured_fp64_peak(torch, dev)

    res = results[headline]
    value = world * B * args.steps / (res["ms"] * 1e-3)
    result = None
    if rank == 0:
        e2e = None
        if not args.no_e2e:
            e2e = e2e_run(gsht, grid, torch, coef_h, headline, args)
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            rr, why = reference_run(L, 1, 0)
            cpu = ({k: rr[k] for k in ("value", "unit", "cores", "kind", "sample",
                                       "single_core_value")}
                   if rr else {"value": None, "unavailable": why})
        mode_lines = {}
        for m in modes:
            r = results[m]
            mode_lines[m] = {
                "value": world * B * args.steps / (r["ms"] * 1e-3), "unit": UNIT,
                "ms_per_step": r["ms"] / args.steps,
                "round_trip_rel_err": r["round_trip_rel_err"],
                "inverse_rel_err_vs_fp64": r.get("inverse_rel_err_vs_fp64"),
                "forward_rel_err_vs_fp64": r.get("forward_rel_err_vs_fp64"),
                "stages": r["stages"],
                "roofline": legendre_roofline(m, r, args, peaks),
                "clocks": r["clocks"],
            }
            if r.get("trace"):
                mode_lines[m]["trace"] = r["trace"]
        if "fp64" in modes:
            for m in modes:
                mode_lines[m]["speedup_vs_fp64_gpu"] = mode_lines[m]["value"] / mode_lines["fp64"]["value"]
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[headline], "data": "synthetic",
            "config": run_config(args), "precision": headline,
            "roofline": mode_lines[headline]["roofline"], "cpu_baseline": cpu, "e2e": e2e,
            "clocks": res["clocks"], "gpu_launches": res["launches"],
            "round_trip_rel_err": res["round_trip_rel_err"], "modes": mode_lines,
        }
    grid.close()
    if rank == 0:
        if world == 1 and not args.no_secondary:
            result["secondary"] = secondary_workloads(args)
        print(json.dumps(result))
    if world > 1:
        dist.destroy_process_group()
    return 0


def e2e_run(gsht, grid, torch, coef_h, precision, args):
    """The same round trip through the C ABI with HOST coefficient buffers
    (pinned): every step uploads the coefficients, runs inverse + forward and
    reads the result back; the grid stays in device memory."""
    L, B = args.lmax, args.fields
    cin = torch.from_numpy(coef_h).pin_memory()
    cout = torch.zeros_like(cin).pin_memory()
    field = torch.empty((B, grid.FieldSize()), dtype=torch.complex128, device="cuda")
    steps = max(1, min(args.steps, 3))

    # The forward accumulates into cout; it is not cleared between steps
    # (clearing 1 GB of host memory is the caller's work, not the
    # transform's), so after k steps it holds k round trips of cin.
    def step():
        grid.inverse_batch(L, N_UPPER, cin, field, precision)
        grid.forward_batch(L, N_UPPER, field, cout, precision)

    step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    rt_err = float(torch.linalg.norm(cout / (steps + 1) - cin) / torch.linalg.norm(cin))
    nbytes = cin.numel() * 16
    # Transfer floor: plain pinned copies of the same buffers. The uploads
    # (2 x nbytes) are the larger direction; the download overlaps them.
    dev = torch.empty_like(cin, device="cuda")
    for _ in range(2):
        dev.copy_(cin, non_blocking=True)
        cout.copy_(dev, non_blocking=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    dev.copy_(cin, non_blocking=True)
    torch.cuda.synchronize()
    h2d_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    cout.copy_(dev, non_blocking=True)
    torch.cuda.synchronize()
    d2h_s = time.perf_counter() - t1
    del dev
    floor_s = max(2 * h2d_s, d2h_s)
    return {"value": B * steps / dt, "unit": UNIT,
            "h2d_bytes_per_step": 2 * nbytes, "d2h_bytes_per_step": nbytes,
            "round_trip_rel_err": rt_err,
            "pcie": {"h2d_GBps": nbytes / h2d_s / 1e9, "d2h_GBps": nbytes / d2h_s / 1e9,
                     "floor_ms_per_step": floor_s * 1e3, "ms_per_step": dt / steps * 1e3,
                     "frac_of_floor": floor_s / (dt / steps)},
            "note": "host coefficients in and out (pinned), grid resident on the GPU; "
                    "the forward output is uploaded because the forward accumulates into it; "
                    "the library moves host batches in chunks that overlap the transforms"}


# ---------------------------------------------------------------------------
# Further workloads (reported lines; the headline metric is the default run)
# ---------------------------------------------------------------------------
def _event_time(torch, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def impl_batch(args, emit=True):
    """256 fields, lmax uniform in {32, 64, 128, 256, 512}, upper index uniform
    in -2..2, half real; envelope 1/(l+1); each on its own grid. One round
    trip (inverse then forward) of all fields per step: one CUDA graph launch
    of the autotuned batch plan, against per-field single calls."""
    import torch
    import gshtrans_b200 as gsht

    prec = args.precision or "bf16x3"
    rng = np.random.default_rng(2024)
    fields, host = [], []
    for i in range(256):
        lmax = int(rng.choice([32, 64, 128, 256, 512]))
        n = int(rng.integers(-2, 3))
        is_real = i % 2 == 1
        c = gsht.random_coefficients(rng, lmax, lmax, n, is_real, 1.0)
        cin = torch.from_numpy(c).cuda()
        npts = (lmax + 1) * 2 * lmax
        grid = torch.zeros(npts, dtype=torch.float64 if is_real else torch.complex128, device="cuda")
        fields.append((lmax, n, is_real, cin, grid, torch.zeros_like(cin)))
        host.append(c)
    t0 = time.perf_counter()
    batch = gsht.Batch(fields, precision=prec, autotune=True)
    plan_s = time.perf_counter() - t0
    groups, grids, nodes = batch.info()
    ms_graph = _event_time(torch, batch.round_trip, args.steps, args.warmup)
    # per-field single calls on grids built once per degree
    forms = () if prec == "fp64" else (prec,)
    gridobj = {L: gsht.GaussLegendreGrid(L, 2, forms=forms) for L in sorted({f[0] for f in fields})}

    def per_field():
        for lmax, n, is_real, cin, grid, cout in fields:
            g = gridobj[lmax]
            g.InverseTransformation(lmax, n, cin, grid, prec)
            g.ForwardTransformation(lmax, n, grid, cout, prec)

    ms_single = _event_time(torch, per_field, max(1, args.steps // 2), 1)
    # accuracy of one round trip against the FP64 batch
    err = None
    if prec != "fp64":
        outs = [torch.zeros_like(f[5]) for f in fields]
        b2 = gsht.Batch([f[:5] + (o,) for f, o in zip(fields, outs)], precision=prec, autotune=True)
        b2.round_trip()
        outs64 = [torch.zeros_like(f[5]) for f in fields]
        b3 = gsht.Batch([f[:5] + (o,) for f, o in zip(fields, outs64)], precision="fp64", autotune=False)
        b3.round_trip()
        torch.cuda.synchronize()
        num = sum(float(torch.linalg.norm(a - b) ** 2) for a, b in zip(outs, outs64))
        den = sum(float(torch.linalg.norm(b) ** 2) for b in outs64)
        err = (num / den) ** 0.5
        b2.close()
        b3.close()
    for g in gridobj.values():
        g.close()
    tiles = {}
    for lm, n, re, cnt, tile in batch.groups():
        tiles[tile] = tiles.get(tile, 0) + 1
    line = {
        "metric": "batched uneven fields, fwd+inv/s (one CUDA graph per step)",
        "value": 256 / (ms_graph * 1e-3), "unit": UNIT, "ms_per_step": ms_graph,
        "per_field_calls": {"value": 256 / (ms_single * 1e-3), "ms_per_step": ms_single},
        "speedup_vs_per_field_calls": ms_single / ms_graph,
        "precision": prec, "round_trip_rel_err_vs_fp64": err,
        "groups": groups, "grids": grids, "graph_nodes_round_trip": nodes[2],
        "autotuned_tile_widths": tiles, "autotuned_streams": batch.streams(),
        "plan_seconds": plan_s,
        "config": {"workload": "256 fields, lmax in {32,64,128,256,512}, n in -2..2, half real, "
                               "envelope (l+1)^-1, own grid per field", "steps": args.steps,
                   "warmup": args.warmup},
    }
    batch.close()
    if not emit:
        return line
    print(json.dumps(line))
    return 0


def table_rows(L, n):
    na = abs(n)
    return sum(L + 1 - max(m, na) for m in range(L + 1))


def impl_large(args, emit=True):
    """One complex field at lmax 2048 (nTheta 2049, nPhi 4096), n = 1,
    envelope (l+1)^-2: table streaming, reported in GB/s of the stored table
    form read per transform; and the same transforms with the Wigner values
    generated by the l-recurrence inside the contraction (no stored table)."""
    import torch
    import gshtrans_b200 as gsht

    L = 2048 if args.lmax == L_MAX else args.lmax  # --lmax selects a smaller case
    n = 1
    rng = np.random.default_rng(2048)
    c_h = gsht.random_coefficients(rng, L, L, n, False, 2.0)
    # A grid without a table: build time and device memory.
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    t0 = time.perf_counter()
    rgrid = gsht.GaussLegendreGrid(L, n, nrange=gsht.Single, forms=("recurrence",))
    rec_build_s = time.perf_counter() - t0
    rec_bytes = free0 - torch.cuda.mem_get_info()[0]
    t0 = time.perf_counter()
    grid = gsht.GaussLegendreGrid(L, n, nrange=gsht.Single, forms=("ozaki",))
    build_s = time.perf_counter() - t0
    coef = torch.from_numpy(c_h).cuda()
    field = torch.empty(grid.FieldSize(), dtype=torch.complex128, device="cuda")
    out = torch.zeros_like(coef)
    tp = (L + 1 + 15) // 16 * 16
    rows = table_rows(L, n)
    hbm = None
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        hbm = json.load(open(mp)).get("hbm_gbs")
    res = {}
    ref = {}
    fp64_table_bytes = rows * tp * 8
    for prec, bytes_per, g in (("fp64", 8, grid), ("ozaki", 7, grid), ("recurrence", 0, rgrid)):
        table_bytes = rows * tp * bytes_per
        ms_inv = _event_time(torch, lambda: g.InverseTransformation(L, n, coef, field, prec),
                             args.steps, args.warmup)
        ms_fwd = _event_time(torch, lambda: g.ForwardTransformation(L, n, field, out, prec),
                             args.steps, args.warmup)
        f = torch.empty_like(field)
        g.InverseTransformation(L, n, coef, f, prec)
        c = torch.zeros_like(coef)
        g.ForwardTransformation(L, n, f, c, prec)
        torch.cuda.synchronize()
        ref[prec] = (f, c)
        r = {"inverse_ms": ms_inv, "forward_ms": ms_fwd, "table_bytes": table_bytes,
             "round_trip_rel_err": float(torch.linalg.norm(c - coef) / torch.linalg.norm(coef))}
        if table_bytes:
            r["inverse_table_GBps"] = table_bytes / (ms_inv * 1e-3) / 1e9
            r["forward_table_GBps"] = table_bytes / (ms_fwd * 1e-3) / 1e9
            if hbm:
                r["frac_of_measured_hbm"] = max(r["inverse_table_GBps"], r["forward_table_GBps"]) / hbm
        else:
            # FP64 work of the fused kernels per transform: the recurrence
            # step (5 flops) and the contraction of the +m and -m rows
            # (8 flops) per (row, colatitude).
            flops = 13.0 * rows * (L + 1)
            r["inverse_fp64_TFLOPs"] = flops / (ms_inv * 1e-3) / 1e12
            r["forward_fp64_TFLOPs"] = flops / (ms_fwd * 1e-3) / 1e12
            r["speedup_vs_stored_fp64_table"] = ((res["fp64"]["inverse_ms"] + res["fp64"]["forward_ms"])
                                                 / (ms_inv + ms_fwd))
            r["grid_build_seconds"] = rec_build_s
            r["grid_device_bytes"] = rec_bytes
        res[prec] = r
    f64, c64 = ref["fp64"]
    for prec in ("ozaki", "recurrence"):
        fo, co = ref[prec]
        res[prec]["inverse_rel_err_vs_fp64"] = float(torch.linalg.norm(fo - f64) / torch.linalg.norm(f64))
        res[prec]["forward_rel_err_vs_fp64"] = float(torch.linalg.norm(co - c64) / torch.linalg.norm(c64))
    line = {
        "metric": f"lmax {L} single field: table streaming GB/s", "unit": "GB/s",
        "value": res["fp64"]["inverse_table_GBps"], "modes": res, "hbm_peak_GBps": hbm,
        "grid_build_seconds": build_s, "fp64_table_bytes": fp64_table_bytes,
        "config": {"workload": f"1 complex field, lmax {L} (nTheta {L + 1}, nPhi {2 * L}), n=1, "
                               "envelope (l+1)^-2", "table_rows": rows, "theta_pad": tp},
    }
    grid.close()
    rgrid.close()
    if not emit:
        return line
    print(json.dumps(line))
    return 0


def impl_pipeline(args, emit=True):
    """64 pairs (u: n = +1, v: n = -1) at lmax 768 (nPhi 1536 = 2^9 x 3):
    inverse both, w = u v + conj(u) u (the conjugate taken with upper index
    -1, so both terms have n = 0) fused in one kernel, forward w."""
    import torch
    import gshtrans_b200 as gsht
    from gshtrans_b200 import fields as F

    L, B = 768, args.fields
    rng = np.random.default_rng(768)
    U = torch.from_numpy(np.stack([gsht.random_coefficients(rng, L, L, 1, False, 1.5)
                                   for _ in range(B)])).cuda()
    V = torch.from_numpy(np.stack([gsht.random_coefficients(rng, L, L, -1, False, 1.5)
                                   for _ in range(B)])).cuda()
    grid = gsht.GaussLegendreGrid(L, 1, forms=("bf16x3", "ozaki"))
    fs = grid.FieldSize()
    Fu = torch.empty((B, fs), dtype=torch.complex128, device="cuda")
    Fv = torch.empty_like(Fu)
    W = torch.empty_like(Fu)
    Cw = torch.zeros((B, gsht.coefficient_size(L, 0, False)), dtype=torch.complex128, device="cuda")
    u = F.Field(grid, 1, count=B, data=Fu)
    v = F.Field(grid, -1, count=B, data=Fv)
    w = F.Field(grid, 0, count=B, data=W)
    expr = u * v + F.conj(u, upper_index=-1) * u
    out = {}
    for prec in ("fp64", "bf16x3", "ozaki"):
        def step():
            grid.inverse_batch(L, 1, U, Fu, prec)
            grid.inverse_batch(L, -1, V, Fv, prec)
            w.assign(expr)
            Cw.zero_()
            grid.forward_batch(L, 0, W, Cw, prec)

        ms = _event_time(torch, step, args.steps, args.warmup)
        step()
        torch.cuda.synchronize()
        out[prec] = {"ms_per_step": ms, "pairs_per_s": B / (ms * 1e-3), "result": Cw.clone()}
    ref = out["fp64"]["result"]
    for prec in out:
        out[prec]["rel_err_vs_fp64"] = float(torch.linalg.norm(out[prec]["result"] - ref) / torch.linalg.norm(ref))
        del out[prec]["result"]
    for prec in out:
        out[prec]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out[prec]["ms_per_step"]
    # The fused expression kernel alone (k_field_eval): reads u and v once,
    # writes w once; 3 x 16 B per grid point, the 64 x 1.18 M points (3.6 GB
    # per launch) far larger than L2.
    ms_eval = _event_time(torch, lambda: w.assign(expr), max(args.steps, 10), max(args.warmup, 3))
    bytes_eval = 3 * 16 * B * fs
    hbm = None
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        hbm = json.load(open(mp)).get("hbm_gbs")
    gbs = bytes_eval / (ms_eval * 1e-3) / 1e9
    field_eval = {"kernel": "k_field_eval", "ms": ms_eval, "algorithmic_bytes": bytes_eval,
                  "achieved_gbs": gbs, "peak_gbs": hbm,
                  "frac": gbs / hbm if hbm else None,
                  "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}
    line = {
        "metric": "field-product pipeline pairs/s (2 inverses, fused u*v + conj(u)*u, 1 forward)",
        "unit": "pairs/s", "value": out["ozaki"]["pairs_per_s"], "modes": out,
        "field_eval": field_eval,
        "config": {"workload": f"{B} pairs, lmax 768 (nTheta 769, nPhi 1536), u n=+1, v n=-1, "
                               "envelope (l+1)^-1.5", "steps": args.steps, "warmup": args.warmup},
    }
    grid.close()
    if not emit:
        return line
    print(json.dumps(line))
    return 0


def secondary_workloads(args):
    """The other workloads of the task, measured in the same run with a few
    steps each (their own lines come from --workload batch | large |
    pipeline): 256 uneven fields in one graph, one field at lmax 2048, the
    field-product pipeline at lmax 768."""
    import copy

    out = {}
    for name, fn in (("batch", impl_batch), ("large", impl_large), ("pipeline", impl_pipeline)):
        a = copy.copy(args)
        a.steps, a.warmup = 5, 3
        a.precision = None
        a.fields = FIELDS
        try:
            out[name] = fn(a, emit=False)
        except Exception as e:  # report, do not lose the headline line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return impl_reference(args)
    if args.workload == "batch":
        return impl_batch(args)
    if args.workload == "large":
        return impl_large(args)
    if args.workload == "pipeline":
        return impl_pipeline(args)
    return impl_ours(args)


if __name__ == "__main__":
    sys.exit(main())
