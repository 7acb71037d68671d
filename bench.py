#!/usr/bin/env python
"""Benchmark of the KPolaris-B200 RIAF image path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--path mixed|plain] [--n 256] [--batch 8]

Workload: the multi-frequency RIAF configuration -- 256x256 pixels,
frequencies {86, 230, 345, 690} GHz sharing one geodesic per pixel, adaptive
step-doubling RK4 (tolerance 1e-8), Cartesian Kerr-Schild a = 0.9375, observer
at r = 1000 M, inclination 17 deg.  Inputs are the analytic plasma model
(synthetic by construction).

Headline (`--path mixed`, default): one step traces `--batch` images through
kp_batch_riaf, the mixed-precision wavefront engine (FP64 geodesic state and
step control, FP32 far-field contraction and FP32 transfer).  The plain FP64
one-image-per-launch kernel is timed in the same run (`plain_fp64`), and the
first image of the batch is compared with it (`accuracy_vs_fp64`: total flux
and image-integrated EVPA per frequency).  `--path plain` makes the plain
kernel the headline.

Metric: 256^2 images/s (whole job).  `value` is device-timed with outputs in
HBM; `e2e` goes through the public API with pinned host output buffers, job-table
upload and device-to-host copies inside the timed region.  Multi-GPU runs are
independent replicas (weak scaling): no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "256\u00b2 images/s & p50/p99 latency, mixed batched vs plain FP64, \u22641e-4 flux err"
UNIT = "images/s"
FLOP_TABLE = ROOT / "profiles" / "flop_counts.json"
TRAFFIC_TABLE = ROOT / "profiles" / "ncu_traffic.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="mixed", choices=["plain", "mixed"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--batch", type=int, default=8, help="images per step of the mixed path")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed images of the plain FP64 kernel")
    ap.add_argument("--serve-requests", type=int, default=48, help="requests of the serving trace (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate of the trace, 1/s")
    ap.add_argument("--serve-plain", type=int, default=1, help="replay the trace on the plain FP64 kernel too")
    ap.add_argument("--serve-rates", default="5,20,50,100,200",
                    help="arrival rates of the serving curve, 1/s (the trace's arrival times rescaled)")
    ap.add_argument("--ref-row-stride", type=int, default=8,
                    help="reference arm: every N-th image row is traced per step")
    ap.add_argument("--fp64-batched-steps", type=int, default=2,
                    help="timed steps of the FP64 policy of the batched engine (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU-baseline sample")
    ap.add_argument("--grmhd", type=int, default=1,
                    help="also time the GRMHD image (288x128x128 FM torus, 512^2, FP64 and mixed)")
    ap.add_argument("--grmhd-steps", type=int, default=2, help="timed GRMHD images per precision")
    ap.add_argument("--grmhd-only", action="store_true",
                    help="profiling entry: only trace GRMHD images (--grmhd-grid, --grmhd-n, --grmhd-precision, "
                         "--grmhd-steps images) and print their times; no JSON line")
    ap.add_argument("--grmhd-grid", type=int, nargs=3, default=[288, 128, 128])
    ap.add_argument("--grmhd-n", type=int, default=512)
    ap.add_argument("--grmhd-precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--config4", type=int, default=1,
                    help="also time the uneven 64-image batch (autotuned, graph-captured) and the slow-light job")
    ap.add_argument("--analysis", type=int, default=1,
                    help="also time an analysis-mode image (kp_image_riaf_analysis) beside the plain FP64 image")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value, pg=None, device=None):
    """The largest `value` over all ranks (replica timing takes the slowest
    rank); the identity without a process group."""
    if pg is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def workload(n):
    from kpolaris_b200 import configs

    params, model, freqs = configs.config2(n, n)
    return params, model, freqs


def config_dict(n, path, nfreq, world, batch=1):
    return {"workload": f"riaf_{n}x{n}_4freq_adaptive_rk4", "images_per_step": batch,
            "pixels": n * n, "nfreq": nfreq,
            "spin": 0.9375, "inclination_deg": 17.0, "r_obs": 1000.0, "tolerance": 1e-8,
            "path": path, "parallelism": f"replicas{world}",
            "l2": "flushed between timed steps (512 MiB write)",
            "model": "analytic RIAF (synthetic)"}


# ---------------------------------------------------------------- CPU legs
CPU = {"cores": os.cpu_count() or 1, "logical": os.cpu_count() or 1, "pinning": "none"}


def physical_core_first(available, topology_root=Path("/sys/devices/system/cpu")):
    """The allowed logical CPUs ordered one per physical core first, SMT
    siblings after (the reference's CPU benchmark policy,
    scripts/benchmark_image_scaling.py:41-53)."""
    groups = {}
    for cpu in sorted(available):
        base = topology_root / f"cpu{cpu}" / "topology"
        try:
            core = (int((base / "physical_package_id").read_text()), int((base / "core_id").read_text()))
        except (OSError, ValueError):
            core = ("unknown", cpu)
        groups.setdefault(core, []).append(cpu)
    width = max(map(len, groups.values()), default=0)
    return [cpus[i] for i in range(width) for cpus in groups.values() if i < len(cpus)], len(groups)


def pin_physical_cores():
    """Pins this process to one logical CPU per physical core and sets the
    OpenMP environment of the CPU oracles (OMP_NUM_THREADS = physical cores,
    spread over those CPUs), as the reference's benchmark does for its
    OpenMP backend.  Must run before the oracle libraries load."""
    try:
        available = os.sched_getaffinity(0)
    except AttributeError:
        return
    order, ncores = physical_core_first(available)
    chosen = order[:ncores]
    try:
        os.sched_setaffinity(0, chosen)
    except OSError:
        return
    os.environ["OMP_NUM_THREADS"] = str(ncores)
    os.environ["OMP_PROC_BIND"] = "spread"
    os.environ["OMP_PLACES"] = "threads"
    CPU.update(cores=ncores, logical=len(available),
               pinning=f"physical-core-first: {ncores} threads on CPUs {chosen[0]}..{chosen[-1]} "
                       f"({ncores} physical cores, {len(available)} logical CPUs allowed), OMP_PROC_BIND=spread")


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
    cores = threads if threads > 0 else CPU["cores"]
    sample = f"{rows_done} of {ny} rows ({rows_done * nx} pixels, spread over the image), {dt:.2f} s"
    return ips, sample, cores


GRMHD_WORKLOAD = ("FMKS GRMHD image: seeded FM torus (a=0.9375, r_in=6, r_max=12, 10% log-normal density "
                  "noise, one poloidal loop at beta=100, heating 1/r) on 288x128x128 FP32 cells, 512^2 pixels, "
                  "230 GHz, i=163 deg, R-beta R_high=40, Dexter fit, derived scalars on the device, "
                  "M87* 6.5e9 Msun, M_unit=1e27 g, adaptive RK4 tol 1e-8")


def grmhd_section(args, torch, dev, local, stream, flush, rank):
    """The GRMHD image (FMKS metric, grid plasma) in FP64 and mixed precision:
    device time per image with the grid resident and outputs on the device
    (CUDA events on the launching stream, L2 flushed before each image), the
    mixed image's error against the FP64 one, and a bounded CPU sample of the
    reference's own GRMHD path."""
    import numpy as np

    import kpolaris_b200 as kp
    from kpolaris_b200 import _abi, synthetic

    n = 512
    prims, model = synthetic.fm_torus(288, 128, 128)
    model.trat_large = 40.0
    params = synthetic.fmks_pass_a_params(model, n, n)
    freqs = [230.0e9]
    lib = kp.library()
    fa = (C.c_double * 1)(*freqs)
    res = {"workload": GRMHD_WORKLOAD}
    outs = {}
    with kp.Grid(model, prims, device=local) as grid:
        for name, prec in (("fp64", _abi.PRECISION_FP64), ("mixed", _abi.PRECISION_MIXED)):
            opt = kp._options(precision=prec, device=local)
            opt.outputs_on_device = 1
            opt.stream = C.c_void_p(stream.cuda_stream)
            out = device_outputs(torch, n * n, 1, dev)
            kp.check(lib.kp_image_grmhd(C.byref(params), grid._h, 1, fa, 1, C.byref(opt), C.byref(out[0])))
            ms = []
            for _ in range(max(1, args.grmhd_steps)):
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                kp.check(lib.kp_image_grmhd(C.byref(params), grid._h, 1, fa, 1, C.byref(opt), C.byref(out[0])))
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            t = sum(ms) / len(ms)
            img = [x.cpu().numpy()[0] for x in out[1][0]]
            ints = [x.cpu().numpy() for x in out[1][2]]
            steps = int(ints[0].astype("int64").sum() + ints[1].astype("int64").sum())
            outs[name] = (img, ints)
            res[name] = {"images_per_s": 1000.0 / t, "ms_per_image": t, "rays_per_s": n * n * 1000.0 / t,
                         "geodesic_steps_per_s": steps * 1000.0 / t,
                         "flux_jy": synthetic.flux_jy(img[0], freqs[0], 20.0, n, n)}
    (a, ai), (b, bi) = outs["fp64"], outs["mixed"]
    ia, ib = integrated_stokes(a[0][None], a[1][None], a[2][None])[0], integrated_stokes(b[0][None], b[1][None], b[2][None])[0]
    res["mixed_vs_fp64"] = {"total_flux_rel_err": abs(ib[0] / ia[0] - 1.0),
                            "evpa_err_deg": abs((ib[1] - ia[1] + 90.0) % 180.0 - 90.0),
                            "reason_agreement": float(np.mean(ai[2] == bi[2]))}
    res["speedup_mixed_vs_fp64"] = res["mixed"]["images_per_s"] / res["fp64"]["images_per_s"]
    if rank == 0:
        import oracle

        if oracle.ref_available():
            derived = oracle.grmhd_derived(model, prims)
            host = _abi.ImageHostData.allocate(n * n, 1)
            rows, t0 = 0, time.perf_counter()
            order = [j for off in range(16) for j in range(off, n, 16)]
            for j in order:
                oracle.image_grmhd(params, model, prims, derived, freqs, threads=0, pixel_begin=j * n,
                                   pixel_end=(j + 1) * n, out=host)
                rows += 1
                if time.perf_counter() - t0 >= args.cpu_seconds:
                    break
            dt = time.perf_counter() - t0
            ips = rows * n / float(n * n) / dt
            res["cpu_baseline"] = {"value": ips, "unit": "images/s", "cores": os.cpu_count() or 1,
                                   "kind": "reference",
                                   "sample": f"{rows} of {n} rows ({rows * n} pixels, spread over the image), "
                                             f"{dt:.2f} s, FP64, derived scalars precomputed"}
    return res


def analysis_section(args, local, flush, torch, rank):
    """Analysis mode: one 256^2 single-frequency (230 GHz) RIAF image with the
    line-of-sight diagnostics (16 radial bins), config-2 controls, through
    kp_image_riaf_analysis with host outputs (device time plus the copies of
    the image and 52 analysis arrays), beside the plain FP64 image of the
    same frequency; the reference's own analysis code on a bounded CPU
    sample of the same image."""
    import kpolaris_b200 as kp
    from kpolaris_b200 import _abi, configs

    n = 256
    params, model, _ = configs.config2(n, n)
    cfg = _abi.default_analysis_config()
    kp.image_riaf_analysis(params, model, cfg, device=local)
    times, plain = [], []
    for _ in range(2):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        kp.image_riaf_analysis(params, model, cfg, device=local)
        times.append(time.perf_counter() - t0)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        kp.image_riaf(params, model, [model.freq_cgs], device=local)
        plain.append(time.perf_counter() - t0)
    res = {"workload": "RIAF 256^2, 230 GHz, config-2 controls (adaptive RK4 tol 1e-8), analysis mode with "
                       "16 logarithmic radial bins 2-100 M, FP64 per-pixel kernel",
           "seconds_incl_d2h": min(times), "images_per_s": 1.0 / min(times),
           "plain_fp64_seconds_incl_d2h": min(plain)}
    if rank == 0:
        import oracle

        if oracle.ref_available():
            host = _abi.ImageHostData.allocate(n * n, 1)
            an = _abi.AnalysisHostData.allocate(n * n, int(cfg.radial_bins))
            rows, t0 = 0, time.perf_counter()
            for j in [j for off in range(16) for j in range(off, n, 16)]:
                oracle.image_riaf_analysis(params, model, cfg, threads=0, pixel_begin=j * n,
                                           pixel_end=(j + 1) * n, out=host, analysis=an)
                rows += 1
                if time.perf_counter() - t0 >= min(args.cpu_seconds, 6.0):
                    break
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": rows / float(n) / dt, "unit": "images/s", "cores": os.cpu_count() or 1,
                                   "kind": "reference",
                                   "sample": f"{rows} of {n} rows ({rows * n} pixels, spread over the image), "
                                             f"{dt:.2f} s, FP64"}
    return res


def config4_section(local, stream, flush, torch):
    """The uneven batch: 64 seeded RIAF images (32^2..512^2, spins U[0, 0.99],
    inclinations U[10, 170] deg, 1-4 frequencies) in one persistent launch,
    schedule autotuned on a 1/4-resolution sample (the launch loop replayed
    as a CUDA graph when the tuner adopts a graph schedule; device time from
    the library's events, L2 flushed first), beside the untuned eager
    schedule; plus the slow-light
    job (16 resident snapshots of the torus 10 M apart, 256^2)."""
    from contextlib import ExitStack

    import kpolaris_b200 as kp
    from kpolaris_b200 import _abi, configs, synthetic

    jobs = configs.config4_jobs()
    rays = sum(p.camera.nx * p.camera.ny for p, _, _ in jobs)
    ray_freqs = sum(p.camera.nx * p.camera.ny * len(f) for p, _, f in jobs)
    outs = [_abi.ImageHostData.allocate(p.camera.nx * p.camera.ny, len(f)) for p, _, f in jobs]
    res = {"workload": "64 seeded RIAF images, resolutions {32,64,128,256,512}^2, spin U[0,0.99], "
                       "inclination U[10,170] deg, 1-4 of {86,230,345,690} GHz, adaptive RK4 tol 1e-8, mixed",
           "images": len(jobs), "rays": rays, "ray_frequencies": ray_freqs}

    def timed(schedule):
        st = _abi.BatchStats()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        kp.batch_riaf(jobs, outs=outs, precision=_abi.PRECISION_MIXED, schedule=schedule, stats=st, device=local)
        return st.kernel_seconds, st.launches

    timed(_abi.SCHEDULE_PERSISTENT)
    eager_s, eager_launches = timed(_abi.SCHEDULE_PERSISTENT)
    tuning = kp.autotune_batch(configs.config4_jobs(scale=4), precision=_abi.PRECISION_MIXED, device=local)
    # the tuner keeps the eager schedule unless a graph schedule won clearly
    tuned_schedule = _abi.SCHEDULE_GRAPH if tuning.graph_cycles > 0 else _abi.SCHEDULE_PERSISTENT
    timed(tuned_schedule)
    tuned_s, tuned_launches = timed(tuned_schedule)
    res["tuned"] = {"schedule": "graph" if tuning.graph_cycles > 0 else "persistent", "seconds": tuned_s,
                    "images_per_s": len(jobs) / tuned_s, "rays_per_s": rays / tuned_s, "launches": tuned_launches}
    res["persistent_default"] = {"seconds": eager_s, "images_per_s": len(jobs) / eager_s,
                                 "rays_per_s": rays / eager_s, "launches": eager_launches}
    if tuning.graph_cycles == 0:
        # the launch loop as a CUDA graph (default CTAs and cycles), as config 4 names it
        timed(_abi.SCHEDULE_GRAPH)
        graph_s, graph_launches = timed(_abi.SCHEDULE_GRAPH)
        res["graph_default"] = {"seconds": graph_s, "images_per_s": len(jobs) / graph_s,
                                "rays_per_s": rays / graph_s, "launches": graph_launches}
    res["autotune"] = {"sample": "the same 64 jobs at 1/4 resolution",
                       "blocks_per_sm": list(tuning.blocks_per_sm), "graph_cycles": tuning.graph_cycles,
                       "candidates": tuning.candidates, "sample_seconds": tuning.seconds,
                       "sample_default_seconds": tuning.default_seconds}
    # slow-light job
    prims, model, times = synthetic.fm_torus_series(288, 128, 128, count=16, dt=10.0)
    model.trat_large = 40.0
    params = synthetic.fmks_pass_a_params(model, 256, 256)
    with ExitStack() as stack:
        grids = [stack.enter_context(kp.Grid(model, p, device=local)) for p in prims]
        out = {}
        for name, prec in (("fp64", _abi.PRECISION_FP64), ("mixed", _abi.PRECISION_MIXED)):
            kp.image_grmhd_slow_light(params, grids, times, 1100.0, [230e9], precision=prec,
                                      schedule=_abi.SCHEDULE_GRAPH, device=local)
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            img = kp.image_grmhd_slow_light(params, grids, times, 1100.0, [230e9], precision=prec,
                                            schedule=_abi.SCHEDULE_GRAPH, device=local)
            dt = time.perf_counter() - t0
            out[name] = {"seconds_incl_d2h": dt, "flux_jy": synthetic.flux_jy(img.image_i[0], 230e9, 20.0, 256, 256),
                         "reached_camera": int((img.reason == 1).sum()),
                         "time_exhausted": int((img.reason == 6).sum())}
    res["slow_light"] = {"workload": "16 snapshots of the 288x128x128 torus 10 M apart, all resident (5.4 GB), "
                                     "256^2, 230 GHz, t_obs = 1100 M, graph schedule", **out}
    return res


def reference_rows(ny, stride=8):
    """The image rows one reference-arm step traces: every `stride`-th row,
    offset to the middle of its band, the same rows every step."""
    return list(range(stride // 2, ny, stride))


def reference_arm(args):
    """The reference's own CPU implementation of the path (oracle/_ref: its
    hot-path templates, OpenMP dynamic over pixels, all physical cores).
    Each step traces a fixed sample of the benchmark image -- the same
    `--ref-row-stride`-spaced rows every step -- and is timed by wall clock;
    ms_per_step is that time, value the image fraction traced per second."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    from kpolaris_b200 import _abi

    params, model, freqs = workload(args.n)
    kind = "reference" if oracle.ref_available() else "port"
    nx, ny = params.camera.nx, params.camera.ny
    rows = reference_rows(ny, args.ref_row_stride)
    out = _abi.ImageHostData.allocate(nx * ny, len(freqs))
    import numpy as np

    pixels = np.concatenate([np.arange(j * nx, (j + 1) * nx) for j in rows]).astype(np.int32)

    def step():
        t0 = time.perf_counter()
        if kind == "reference":
            # one dynamic loop over every pixel of the sample
            oracle.image_riaf_pixels(params, model, freqs, pixels, threads=0, out=out)
        else:
            for j in rows:
                oracle.image_riaf(params, model, freqs, kind=kind, threads=0, pixel_begin=j * nx,
                                  pixel_end=(j + 1) * nx, out=out)
        return time.perf_counter() - t0

    for _ in range(max(0, args.warmup)):
        step()
    step_s = [step() for _ in range(args.steps)]
    mean_s = sum(step_s) / len(step_s)
    frac = len(rows) / float(ny)
    value = frac / mean_s
    sample = (f"{len(rows)} of {ny} rows per step (every {args.ref_row_stride}th, from row {rows[0]}; "
              f"{len(rows) * nx} pixels = {frac:.4f} image) in one OpenMP dynamic loop, the same rows every "
              f"step, wall clock; "
              f"{CPU['pinning']}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic RIAF plasma)",
        # the workload of the GPU arm (its config); each step is a bounded
        # sample of it, described in cpu_baseline.sample and reference_step
        "config": config_dict(args.n, args.path, len(freqs), world, args.batch),
        "reference_step": {"path": "reference CPU (OpenMP dynamic over pixels)", "image_fraction": frac,
                           "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": CPU["cores"], "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_s": {"min": min(step_s), "max": max(step_s)},
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
    """Algorithmic operation counts of one image of this workload, from the
    committed count of the reference algorithm (oracle/flop_count.cpp)."""
    if not FLOP_TABLE.exists():
        return None
    table = json.loads(FLOP_TABLE.read_text())
    return table.get(f"riaf_{n}x{n}_4freq_adaptive_rk4")


PHASES = ("far", "near_a", "near_b")


def phase_ops(flops, phase, mixed):
    """(fp64_ops, fp32_ops) of one image in one engine phase.  Mixed policy:
    the far phase contracts the connection in FP32 and near-B evaluates the
    plasma and the thermal fits in FP32; the rest is FP64."""
    ph = flops[f"phase_{phase}"]
    rhs, other = ph["rhs_ops"], ph["other_ops"]
    rad = flops["plasma_ops"] + flops["thermal_ops"] if phase == "near_b" else 0
    if not mixed:
        return rhs + other + rad, 0
    if phase == "far":
        return other, rhs
    return rhs + other, rad


def integrated_stokes(i, q, u):
    """Total flux and EVPA (degrees) of each frequency of an image."""
    import numpy as np

    out = []
    for f in range(i.shape[0]):
        ti, tq, tu = float(i[f].sum()), float(q[f].sum()), float(u[f].sum())
        out.append((ti, 0.5 * float(np.degrees(np.arctan2(tu, tq)))))
    return out


# ---------------------------------------------------------------- serving
def serving_trace(n_requests, rate, seed=2026, grmhd_fraction=0.25, ngrids=4):
    """Seeded Poisson arrivals of image requests: resolution 64^2, 128^2 or
    256^2, 1-4 frequencies from {86, 230, 345, 690} GHz, inclination
    U[10, 170] deg, the adaptive 4-frequency controls; a fraction of them
    GRMHD images of one of `ngrids` resident torus grids, the rest RIAF
    images with spin U[0, 0.99].  Entries: (t, kind, params, model or grid
    index, frequencies)."""
    import numpy as np

    from kpolaris_b200 import configs, synthetic

    rng = np.random.default_rng(seed)
    _, gmodel = synthetic.fm_torus(8, 8, 8)
    t = 0.0
    trace = []
    for _ in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice([64, 128, 256]))
        nf = int(rng.integers(1, 5))
        freqs = sorted(rng.choice(configs.CONFIG2_FREQS, size=nf, replace=False).tolist())
        inc = float(rng.uniform(10.0, 170.0))
        if rng.uniform() < grmhd_fraction:
            p = synthetic.fmks_pass_a_params(gmodel, n, n, inclination_deg=inc)
            trace.append((t, "grmhd", p, int(rng.integers(0, ngrids)), freqs))
            continue
        p = configs.riaf_params(n, n, spin=float(rng.uniform(0.0, 0.99)), inclination_deg=inc, step=0.025,
                                adaptive=1, max_steps=400000, adaptive_tolerance=1e-8, min_step=1e-10,
                                max_step=2.0, max_radiation_step=2.0, max_radiation_depth=1.0,
                                max_absorption_depth=1.0, max_faraday_depth=4.0)
        trace.append((t, "riaf", p, configs.riaf_model(), freqs))
    return trace


def serving_grids(device, ngrids=4):
    """The resident grids of the serving trace: 288x128x128 tori, seeds
    2026 + k, R_high = 40."""
    import kpolaris_b200 as kp
    from kpolaris_b200 import synthetic

    grids = []
    for k in range(ngrids):
        prims, model = synthetic.fm_torus(288, 128, 128, seed=2026 + k)
        model.trat_large = 40.0
        grids.append(kp.Grid(model, prims, device=device))
    return grids


def serve_mixed(trace, grids, device):
    """Replays the trace against the serving loop in real time."""
    import kpolaris_b200 as kp

    def submit(srv, kind, p, m, f):
        return srv.submit_grmhd(p, grids[m], f) if kind == "grmhd" else srv.submit(p, m, f)

    with kp.Server(device=device, max_rays=1 << 21) as srv:
        # warm the kernels and the server's buffers with one request of each kind
        for kind in ("riaf", "grmhd"):
            first = next((e for e in trace if e[1] == kind), None)
            if first:
                w = submit(srv, *first[1:])
                srv.wait(w, timeout=120.0)
                srv.result(w)
        base = srv.stats()
        t0 = time.perf_counter()
        tickets = []
        for (t, kind, p, m, f) in trace:
            delay = t - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(submit(srv, kind, p, m, f))
        for tk in tickets:
            srv.wait(tk, timeout=300.0)
        t_end = time.perf_counter()
        st = srv.stats()
    # per-request latency from the server's own clock (submit -> done)
    return {"images_per_s": len(trace) / (t_end - t0), "p50_s": st.latency_p50, "p99_s": st.latency_p99,
            "max_s": st.latency_max, "queue_p50_s": st.queue_p50,
            "max_inflight_jobs": st.max_inflight_jobs, "ticks": st.ticks - base.ticks}


def plain_service_times(trace, grids, device):
    """Service time of every request of the trace on the plain FP64 path
    (RIAF: the one-image-per-launch kernel; GRMHD: one FP64 image per call),
    each measured alone after a warm-up request of each kind."""
    import kpolaris_b200 as kp

    def run(kind, p, m, f):
        if kind == "grmhd":
            kp.image_grmhd(p, grids[m], f, device=device)
        else:
            kp.image_riaf(p, m, f, device=device)

    for kind in ("riaf", "grmhd"):
        first = next((e for e in trace if e[1] == kind), None)
        if first:
            run(*first[1:])
    svc = []
    for (_, kind, p, m, f) in trace:
        t_a = time.perf_counter()
        run(kind, p, m, f)
        svc.append(time.perf_counter() - t_a)
    return svc


def fifo_latency(arrivals, svc):
    """A FIFO of plain launches: each request starts when it has arrived and
    the previous one has finished; a request's service time does not depend
    on when it starts, so one measured set of service times serves every
    arrival rate."""
    import numpy as np

    finish = 0.0
    lat = []
    for t, s in zip(arrivals, svc):
        finish = max(finish, t) + s
        lat.append(finish - t)
    return {"images_per_s": len(arrivals) / finish, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "max_s": float(max(lat)), "busy_s": float(sum(svc))}


def rescale_trace(trace, factor):
    """The trace with every arrival time multiplied by `factor`."""
    return [(e[0] * factor,) + tuple(e[1:]) for e in trace]


def serve_plain(trace, grids, device):
    """The same trace through a FIFO of plain FP64 launches."""
    return fifo_latency([e[0] for e in trace], plain_service_times(trace, grids, device))


def progress(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def ours_arm(args):
    import numpy as np
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
    mixed = args.path == "mixed"
    batch = args.batch if mixed else 1
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # ---- headline path: `batch` images per step through kp_batch_riaf
    # (mixed, wavefront engine) or one image per launch (plain FP64)
    opt = kp._options(precision=_abi.PRECISION_MIXED if mixed else _abi.PRECISION_FP64,
                      schedule=_abi.SCHEDULE_PERSISTENT if mixed else _abi.SCHEDULE_PER_PIXEL, device=local)
    opt.outputs_on_device = 1
    opt.stream = C.c_void_p(stream.cuda_stream)
    outs = [device_outputs(torch, npix, nfreq, dev) for _ in range(batch)]
    jobs = (_abi.RiafJob * batch)()
    for b in range(batch):
        j = jobs[b]
        j.params = params
        j.model = model
        for f, v in enumerate(freqs):
            j.frequencies[f] = v
        j.nfreq = nfreq
        j.radiation_substeps = 1
        j.out = outs[b][0]
    fa = (C.c_double * nfreq)(*freqs)
    stats = _abi.BatchStats()
    phase_s = [0.0, 0.0, 0.0]
    launches = [0]

    def step(record=False):
        if mixed:
            kp.check(lib.kp_batch_riaf(jobs, batch, C.byref(opt), C.byref(stats)))
            if record:
                for k in range(3):
                    phase_s[k] += stats.phase_seconds[k]
                launches[0] += stats.launches
        else:
            kp.check(lib.kp_image_riaf(C.byref(params), C.byref(model), 1, fa, nfreq, C.byref(opt),
                                       C.byref(outs[0][0])))
            if record:
                launches[0] += 1

    progress("warm-up")
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    progress("timed steps")
    peak64 = C.c_double(0.0)
    kp.check(lib.kp_measure_fma_peak(local, 1, C.byref(peak64)))
    peak32 = C.c_double(0.0)
    kp.check(lib.kp_measure_fma_peak(local, 0, C.byref(peak32)))

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
        step(record=True)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if pg:
        pg.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = max_over_ranks(sum(step_ms) / len(step_ms), pg, dev)
    value = world * batch * 1000.0 / ms

    progress("plain FP64 kernel")
    # ---- plain FP64 one-image-per-launch kernel, same run, same timing rules
    plain_out = device_outputs(torch, npix, nfreq, dev)
    opt_plain = kp._options(precision=_abi.PRECISION_FP64, schedule=_abi.SCHEDULE_PER_PIXEL, device=local)
    opt_plain.outputs_on_device = 1
    opt_plain.stream = C.c_void_p(stream.cuda_stream)

    def plain_step():
        kp.check(lib.kp_image_riaf(C.byref(params), C.byref(model), 1, fa, nfreq, C.byref(opt_plain),
                                   C.byref(plain_out[0])))

    plain_step()
    plain_ms = []
    for _ in range(args.plain_steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
    plain_img_ms = sum(plain_ms) / len(plain_ms)

    # accuracy of the headline path against the FP64 image (first image)
    img = [t.cpu().numpy() for t in outs[0][1][0]]
    ref = [t.cpu().numpy() for t in plain_out[1][0]]
    got_int = integrated_stokes(img[0], img[1], img[2])
    ref_int = integrated_stokes(ref[0], ref[1], ref[2])
    flux_err = [abs(g[0] / r[0] - 1.0) if r[0] > 0 else 0.0 for g, r in zip(got_int, ref_int)]
    evpa_err = [abs((g[1] - r[1] + 90.0) % 180.0 - 90.0) for g, r in zip(got_int, ref_int)]
    reason_match = float(np.mean(outs[0][1][2][2].cpu().numpy() == plain_out[1][2][2].cpu().numpy()))

    # ---- the FP64 policy of the same batched engine on the same step: splits
    # the speed-up over the plain kernel into engine and precision
    fp64_batched = None
    if mixed and args.fp64_batched_steps > 0:
        progress("FP64 policy of the batched engine")
        opt64 = kp._options(precision=_abi.PRECISION_FP64, schedule=_abi.SCHEDULE_PERSISTENT, device=local)
        opt64.outputs_on_device = 1
        opt64.stream = C.c_void_p(stream.cuda_stream)
        stats64 = _abi.BatchStats()
        kp.check(lib.kp_batch_riaf(jobs, batch, C.byref(opt64), C.byref(stats64)))
        torch.cuda.synchronize()
        b64_ms = []
        for _ in range(args.fp64_batched_steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            kp.check(lib.kp_batch_riaf(jobs, batch, C.byref(opt64), C.byref(stats64)))
            e1.record(stream)
            torch.cuda.synchronize()
            b64_ms.append(e0.elapsed_time(e1))
        b64 = sum(b64_ms) / len(b64_ms)
        same = all(torch.equal(a, b) for a, b in zip(outs[0][1][0], plain_out[1][0]))
        fp64_batched = {"images_per_s": world * batch * 1000.0 / b64, "ms_per_step": b64, "images_per_step": batch,
                        "steps": args.fp64_batched_steps,
                        "stokes_bit_identical_to_plain": bool(same),
                        "path": "kp_batch_riaf, FP64 policy (wavefront engine, the reference's arithmetic)"}


    progress("e2e")
    # ---- e2e: the same batch through the public API with host buffers in
    # pinned memory (the library copies each output array device-to-host)
    pinned = []

    def pinned_host_data():
        arrays = {}
        shapes = [(name, (nfreq, npix), torch.float64) for name in _abi.IMAGE_FIELDS]
        shapes += [(name, (npix,), torch.float64) for name in _abi.DIAG_FIELDS]
        shapes += [(name, (npix,), torch.int32) for name in _abi.INT_FIELDS]
        for name, shape, dt in shapes:
            t = torch.zeros(shape, dtype=dt, pin_memory=True)
            pinned.append(t)
            arrays[name] = t.numpy()
        return _abi.ImageHostData(npix=npix, nfreq=nfreq, arrays=arrays)

    host = [pinned_host_data() for _ in range(batch)]
    job_list = [(params, model, freqs)] * batch
    e2e_ms = []
    for i in range(args.steps + 1):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if mixed:
            kp.batch_riaf(job_list, outs=host, precision=_abi.PRECISION_MIXED, device=local)
        else:
            kp.image_riaf(params, model, freqs, out=host[0], device=local)
        dt = (time.perf_counter() - t0) * 1000.0
        if i > 0:
            e2e_ms.append(dt)
    e2e = max_over_ranks(sum(e2e_ms) / len(e2e_ms), pg, dev)
    d2h = batch * int(lib.kp_image_output_bytes(npix, nfreq))
    h2d = batch * int(lib.kp_abi_sizeof(6))

    steps_per_image = int(host[0].pass_a_steps.astype("int64").sum() + host[0].steps.astype("int64").sum())
    flops = flop_model(args.n)
    roof = None
    phases = None
    if flops and mixed and sum(phase_s) > 0:
        phases = {}
        for k, name in enumerate(PHASES):
            f64, f32 = phase_ops(flops, name, mixed)
            sec = phase_s[k] / args.steps
            phases[name] = {"ms_per_step": sec * 1e3, "share": phase_s[k] / sum(phase_s),
                            "fp64_tflops": batch * f64 / sec / 1e12 if sec > 0 else None,
                            "fp32_tflops": batch * f32 / sec / 1e12 if sec > 0 else None}
        top = max(range(3), key=lambda k: phase_s[k])
        name = PHASES[top]
        f64, f32 = phase_ops(flops, name, mixed)
        sec = phase_s[top] / args.steps
        bound64 = f64 / peak64.value >= f32 / peak32.value
        achieved = batch * (f64 if bound64 else f32) / sec / 1e12
        peak = peak64.value if bound64 else peak32.value
        traffic = None
        if TRAFFIC_TABLE.exists() and args.n == 256 and batch == 8:
            t = json.loads(TRAFFIC_TABLE.read_text()).get(f"wave_{name}_mixed")
            traffic = t["bytes_per_bench_step"] if t else None
        roof = {"bound": "fp64" if bound64 else "fp32", "kernel": f"wave_{name}_mixed",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic,
                "traffic_unit": "DRAM bytes of the phase's launches in one step (ncu, scaled by rays; see profiles/)",
                "peak_source": "measured FMA throughput of this GPU (kp_measure_fma_peak), of measured",
                "flops_source": "algorithmic op count of the reference algorithm per phase "
                                "(profiles/flop_counts.json) x images per launch; the mixed kernels execute "
                                "fewer: the factored contraction, ~320 of the 1080 ops per RHS"}
    elif flops and not mixed:
        achieved = flops["fp64_flops"] / (ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "kernel": "image_fp64_per_pixel", "achieved": achieved,
                "peak": peak64.value, "unit": "TFLOP/s", "frac": achieved / peak64.value, "traffic": None,
                "peak_source": "measured FP64 FMA throughput of this GPU (kp_measure_fma_peak), of measured",
                "flops_source": "algorithmic FP64 op count of the reference algorithm"}

    # the serving trace, config 3 and config 4 are single-GPU measurements:
    # they run at N = 1 only, so replica runs time the headline alone
    serving = None
    if mixed and args.serve_requests > 0 and world == 1:
        progress("serving trace")
        trace = serving_trace(args.serve_requests, args.serve_rate)
        grids = serving_grids(local)
        try:
            serving = {"workload": "Poisson arrivals: 3/4 RIAF images (spin U[0,0.99]), 1/4 GRMHD images of one of "
                                   "4 resident 288x128x128 tori; 64^2/128^2/256^2, 1-4 frequencies, inclination "
                                   "U[10,170] deg, adaptive RK4",
                       "requests": len(trace), "grmhd_requests": sum(1 for e in trace if e[1] == "grmhd"),
                       "rate_per_s": args.serve_rate,
                       "mixed_batched": serve_mixed(trace, grids, local)}
            svc = None
            if args.serve_plain:
                progress("serving trace on the plain FP64 path")
                svc = plain_service_times(trace, grids, local)
                serving["plain_fp64"] = fifo_latency([e[0] for e in trace], svc)
            # the serving curve: the same requests, arrival times rescaled
            curve = []
            for rate in [float(x) for x in args.serve_rates.split(",") if x.strip()]:
                progress(f"serving curve at {rate:g}/s")
                scaled = rescale_trace(trace, args.serve_rate / rate)
                row = {"rate_per_s": rate,
                       "mixed_batched": (serving["mixed_batched"] if rate == args.serve_rate
                                         else serve_mixed(scaled, grids, local))}
                if svc is not None:
                    row["plain_fp64"] = fifo_latency([e[0] for e in scaled], svc)
                curve.append(row)
            serving["curve"] = curve
        finally:
            for g in grids:
                g.release()

    grmhd = None
    if args.grmhd and world == 1:
        progress("GRMHD image")
        grmhd = grmhd_section(args, torch, dev, local, stream, flush, rank)

    config4 = None
    if args.config4 and world == 1:
        progress("uneven batch and slow light")
        config4 = config4_section(local, stream, flush, torch)

    analysis = None
    if args.analysis and world == 1:
        progress("analysis-mode image")
        analysis = analysis_section(args, local, flush, torch, rank)

    cpu = None
    if rank == 0:
        import oracle

        kind = "reference" if oracle.ref_available() else "port"
        v, sample, cores = cpu_sample(params, model, freqs, kind, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": f"{sample}; {CPU['pinning']}"}

    if rank == 0:
        srt = sorted(step_ms)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64-geometry/f32-transfer" if mixed else "f64",
            "data": "synthetic (analytic RIAF plasma)",
            "config": config_dict(args.n, args.path, nfreq, world, batch),
            "e2e": {"value": world * batch * 1000.0 / e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches[0],
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            # the secondary workloads (bulky) before the headline comparison
            # (plain FP64, speed-up, accuracy, latency), which closes the line
            "serving": serving,
            "grmhd": grmhd,
            "config4": config4,
            "analysis": analysis,
            "phases": phases,
            "rays_per_s": value * npix,
            "geodesic_steps_per_s": value * steps_per_image,
            "step_latency_ms": {"p50": float(np.percentile(srt, 50)), "p99": float(np.percentile(srt, 99))},
            "latency_ms": ({"p50": serving["mixed_batched"]["p50_s"] * 1e3,
                            "p99": serving["mixed_batched"]["p99_s"] * 1e3, "source": "serving trace"}
                           if serving else None),
            "accuracy_vs_fp64": {"total_flux_rel_err": flux_err, "evpa_err_deg": evpa_err,
                                 "reason_agreement": reason_match,
                                 "frequencies_ghz": [f * 1e-9 for f in freqs]},
            "plain_fp64": {"images_per_s": world * 1000.0 / plain_img_ms, "ms_per_image": plain_img_ms,
                           "kernel": "image_fp64_per_pixel (one image per launch)"},
            "fp64_batched": fp64_batched,
            "speedup_vs_plain_fp64": value / (world * 1000.0 / plain_img_ms),
        }
        if fp64_batched:
            # engine gain (FP64 batched / plain) x precision gain (mixed / FP64 batched)
            line["speedup_split"] = {
                "engine": fp64_batched["images_per_s"] / (world * 1000.0 / plain_img_ms),
                "precision": value / fp64_batched["images_per_s"]}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def grmhd_only(args):
    """Profiling entry: GRMHD images of the seeded torus, nothing else."""
    import numpy as np

    import kpolaris_b200 as kp
    from kpolaris_b200 import _abi, synthetic

    n1, n2, n3 = args.grmhd_grid
    prims, model = synthetic.fm_torus(n1, n2, n3)
    model.trat_large = 40.0
    prec = _abi.PRECISION_MIXED if args.grmhd_precision == "mixed" else _abi.PRECISION_FP64
    params = synthetic.fmks_pass_a_params(model, args.grmhd_n, args.grmhd_n)
    with kp.Grid(model, prims) as g:
        for _ in range(max(1, args.grmhd_steps)):
            t0 = time.perf_counter()
            r = kp.image_grmhd(params, g, [230e9], precision=prec)
            dt = time.perf_counter() - t0
            digest = hashlib.sha256(b"".join(np.ascontiguousarray(r.arrays[k]).tobytes()
                                             for k in sorted(r.arrays))).hexdigest()[:16]
            print(f"grmhd {n1}x{n2}x{n3} {args.grmhd_n}^2 {args.grmhd_precision}: "
                  f"{dt:.3f} s, steps A {int(r.pass_a_steps.sum())} B {int(r.steps.sum())}, image {digest}",
                  flush=True)
    return 0


def main():
    args = parse()
    pin_physical_cores()
    if args.grmhd_only:
        return grmhd_only(args)
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
