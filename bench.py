#!/usr/bin/env python
"""Benchmark of the KPolaris-B200 RIAF image path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--path plain|mixed] [--n 256]

Workload (default): the multi-frequency RIAF configuration -- 256x256 pixels,
frequencies {86, 230, 345, 690} GHz sharing one geodesic per pixel, adaptive
step-doubling RK4 (tolerance 1e-8), Cartesian Kerr-Schild a = 0.9375, observer
at r = 1000 M, inclination 17 deg.  Inputs are the analytic plasma model
(synthetic by construction); one step renders one image on every rank.

Metric: 256^2 images/s (whole job).  `value` is device-timed with outputs in
HBM; `e2e` goes through the C ABI with host output buffers, launch-parameter
upload and device-to-host copies inside the timed region.  Multi-GPU runs are
independent replicas (weak scaling): no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "256^2 images/s (RIAF, 4 frequencies, adaptive RK4)"
UNIT = "images/s"
FLOP_TABLE = ROOT / "profiles" / "flop_counts.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU-baseline sample")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(n):
    from kpolaris_b200 import configs

    params, model, freqs = configs.config2(n, n)
    return params, model, freqs


def config_dict(n, path, nfreq, world):
    return {"workload": f"riaf_{n}x{n}_4freq_adaptive_rk4", "pixels": n * n, "nfreq": nfreq,
            "spin": 0.9375, "inclination_deg": 17.0, "r_obs": 1000.0, "tolerance": 1e-8,
            "path": path, "parallelism": f"replicas{world}",
            "l2": "flushed between timed steps (512 MiB write)",
            "model": "analytic RIAF (synthetic)"}


# ---------------------------------------------------------------- CPU legs
def cpu_sample(params, model, freqs, kind, seconds, threads=0):
    """Times the CPU oracle on evenly spaced image rows until `seconds` of
    wall time are spent (at least one row); returns (images/s, sample text,
    threads used)."""
    import oracle

    nx, ny = params.camera.nx, params.camera.ny
    order = []
    stride = 8
    for off in range(stride):
        order.extend(range(off, ny, stride))
    rows_done = 0
    t0 = time.perf_counter()
    from kpolaris_b200 import _abi
    out = _abi.ImageHostData.allocate(nx * ny, len(freqs))
    for j in order:
        oracle.image_riaf(params, model, freqs, kind=kind, threads=threads, pixel_begin=j * nx,
                          pixel_end=(j + 1) * nx, out=out)
        rows_done += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    frac = rows_done * nx / float(nx * ny)
    ips = frac / dt
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    sample = f"{rows_done} of {ny} rows ({rows_done * nx} pixels, spread over the image), {dt:.2f} s"
    return ips, sample, cores


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle

    params, model, freqs = workload(args.n)
    kind = "reference" if oracle.ref_available() else "port"
    if kind == "reference":
        oracle.lib("reference")
    for _ in range(max(0, args.warmup)):
        cpu_sample(params, model, freqs, kind, seconds=0.0)
    vals = []
    samples = []
    per = max(2.0, args.cpu_seconds / max(1, args.steps))
    cores = os.cpu_count() or 1
    for _ in range(args.steps):
        v, s, cores = cpu_sample(params, model, freqs, kind, seconds=per)
        vals.append(v)
        samples.append(s)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic RIAF plasma)",
        "config": config_dict(args.n, "reference CPU (OpenMP dynamic over pixels)", len(freqs), 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": samples[-1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU leg
class ClockSampler:
    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"kp_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            if self.uuid and self.uuid not in parts[1]:
                continue
            rows.append(parts)
        if not rows:
            return None
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def device_outputs(torch, npix, nfreq, dev):
    from kpolaris_b200 import _abi

    img = [torch.empty((nfreq, npix), dtype=torch.float64, device=dev) for _ in range(4)]
    diag = [torch.empty(npix, dtype=torch.float64, device=dev) for _ in range(11)]
    ints = [torch.empty(npix, dtype=torch.int32, device=dev) for _ in range(3)]
    s = _abi.ImageOut()
    s.npix, s.nfreq = npix, nfreq
    for name, t in zip(_abi.IMAGE_FIELDS, img):
        setattr(s, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)))
    for name, t in zip(_abi.DIAG_FIELDS, diag):
        setattr(s, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)))
    for name, t in zip(_abi.INT_FIELDS, ints):
        setattr(s, name, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int32)))
    return s, (img, diag, ints)


def flop_model(n):
    """Algorithmic FP64 operation count of one image of this workload, from
    the committed count of the reference algorithm (oracle/flop_count)."""
    if not FLOP_TABLE.exists():
        return None
    table = json.loads(FLOP_TABLE.read_text())
    return table.get(f"riaf_{n}x{n}_4freq_adaptive_rk4")


def ours_arm(args):
    import torch

    import kpolaris_b200 as kp
    from kpolaris_b200 import _abi

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    lib = kp.library()
    params, model, freqs = workload(args.n)
    npix = args.n * args.n
    nfreq = len(freqs)
    stream = torch.cuda.current_stream()
    opt = kp._options(precision=_abi.PRECISION_MIXED if args.path == "mixed" else _abi.PRECISION_FP64,
                      schedule=_abi.SCHEDULE_PERSISTENT if args.path == "mixed" else _abi.SCHEDULE_PER_PIXEL,
                      device=local)
    opt.outputs_on_device = 1
    opt.stream = C.c_void_p(stream.cuda_stream)
    outs, keep = device_outputs(torch, npix, nfreq, dev)
    fa = (C.c_double * nfreq)(*freqs)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        kp.check(lib.kp_image_riaf(C.byref(params), C.byref(model), 1, fa, nfreq, C.byref(opt),
                                   C.byref(outs)))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    # roofline denominators measured on this GPU
    peak = C.c_double(0.0)
    kp.check(lib.kp_measure_fma_peak(local, 1, C.byref(peak)))
    fp64_peak = peak.value

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.4)
    evs = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if pg:
        pg.barrier()
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    ms = sum(kernel_ms) / len(kernel_ms)
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * 1000.0 / ms

    # e2e: the same image through the public C ABI with host buffers
    host = _abi.ImageHostData.allocate(npix, nfreq)
    opt_h = kp._options(precision=opt.precision, schedule=opt.schedule, device=local)
    e2e_ms = []
    for i in range(args.steps + 1):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        kp.image_riaf(params, model, freqs, out=host, precision=opt.precision,
                      schedule=opt.schedule, device=local)
        dt = (time.perf_counter() - t0) * 1000.0
        if i > 0:
            e2e_ms.append(dt)
    e2e = sum(e2e_ms) / len(e2e_ms)
    if pg:
        t = torch.tensor([e2e], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e = float(t.item())
    d2h = lib.kp_image_output_bytes(npix, nfreq)
    lib.kp_abi_sizeof.restype = C.c_size_t
    h2d = int(lib.kp_abi_sizeof(6))

    steps_per_image = int(host.pass_a_steps.astype("int64").sum() + host.steps.astype("int64").sum())
    flops = flop_model(args.n)
    roof = None
    if flops:
        achieved = flops["fp64_flops"] / (ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": flops.get("dram_bytes_per_launch"),
                "peak_source": "measured FP64 FMA throughput on this GPU (kp_measure_fma_peak)",
                "flops_source": "algorithmic FP64 operation count of the reference algorithm"}

    cpu = None
    if rank == 0:
        import oracle

        kind = "reference" if oracle.ref_available() else "port"
        v, sample, cores = cpu_sample(params, model, freqs, kind, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.path == "plain" else "f64-geometry/f32-transfer",
            "data": "synthetic (analytic RIAF plasma)", "config": config_dict(args.n, args.path, nfreq, world),
            "e2e": {"value": world * 1000.0 / e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps,
            "rays_per_s": value * npix,
            "geodesic_steps_per_s": value * steps_per_image,
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
