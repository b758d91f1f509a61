"""Benchmark: photons/s of the photon-propagation path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload bilayer_rgd_mie] [--photons P] [--precision fp32|fp64]

One step = one transport pass over P photons of the workload (default: the
two-layer RGD-over-Mie slab with FarFieldCBS 200x8, PlanarFluence 200x200x64 and
FarFieldFluence 90x36 detectors, 1e8 photons per step).  `value` is photons/s of
the whole job with tallies resident in HBM, timed with CUDA events on the
launching stream; `e2e` is the same metric through the public API
(run_simulation_parallel with host tally arrays, host<->device copies inside).
Under torchrun each rank transports its own photon range (weak scaling) and rank
0 prints one JSON line with the max-over-ranks time.  `--impl reference` times
the reference's own CPU implementation (built from its sources into oracle/_ref)
on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "luminis-mc_b200"))
sys.path.insert(0, REPO)

FLOP_PER_EVENT = 300        # FP32 flops per scattering event (add/mul = 1, FMA = 2)
# FP32 flops of one (vertex, bin) pair of the estimator-mode FarFieldCBS, counted from the
# reference's per-bin arithmetic (FarFieldCBSSensor::process_estimation,
# src/detector.cpp:1384-1560) for a vertex from the second event on: the exit frame and
# forward field (~185), the reverse path's last stage and its normalisation (~205), the
# CBS phase and reverse field (~30), the Stokes values and their accumulation (~62);
# plus ~13 SFU operations (exp, sqrt, atan2, sincos) not counted.
FLOP_PER_EST_PAIR = 480
METRIC = "photons/s"


def _hbm_peak():
    """Measured HBM copy bandwidth of the B200 (MEASURED_PEAKS.json beside this file),
    else 6.65 TB/s, an earlier STREAM-style copy measurement on B200."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, "fallback: 6.65 TB/s, an earlier B200 copy measurement (MEASURED_PEAKS.json absent)"


HBM_PEAK_GBS = _hbm_peak()
# DRAM bytes (read + write) per photon of one FP32 transport launch on bilayer_rgd_mie
# with CBS replay: 2.41 MB read + 138.82 MB written for a 2 M-photon launch in one ncu
# capture of the transport kernel; the traffic is the hit queue, so it grows with the
# photons.
TRAFFIC_BYTES_PER_PHOTON = {"bilayer_rgd_mie": (2.405120e6 + 138.818048e6) / 2e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bilayer_rgd_mie")
    ap.add_argument("--photons", type=int, default=None)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU work per reference sample (bounded)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--block-size", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--batch-photons", type=int, default=0)
    ap.add_argument("--stage-tables", action="store_true",
                    help="binary32 amplitude tables staged in shared memory (1-D bulk copies)")
    ap.add_argument("--no-replay", action="store_true",
                    help="keep every photon's reverse-path history instead of replaying CBS hits")
    ap.add_argument("--tally-mode", default="default",
                    choices=["default", "global", "warp", "shared"],
                    help="how the hit-queue tally kernel adds into the sensor grids")
    ap.add_argument("--variant-steps", type=int, default=2,
                    help="timed steps of the FP64 and FP32+adjoint variants (0: skip them)")
    ap.add_argument("--variants", default="fp64,differentiable,sweep,estimator,f2,long_paths",
                    help="comma-separated subset of the variant arms to measure")
    ap.add_argument("--estimator-photons", type=int, default=1_000_000,
                    help="photons of the estimator-mode variant")
    ap.add_argument("--precision-report", action="store_true",
                    help="instead of timing: FP32 tallies against FP64 on the same random "
                         "numbers, per sensor, for the named workloads")
    return ap.parse_args()


def workload_spec(name, photons):
    from luminis_mc_b200 import workloads as W
    spec = W.WORKLOADS[name]()
    if photons is not None:
        spec["n_photons"] = int(photons)
    return spec


def config_block(spec, args, n_gpus):
    return {"workload": spec["name"], "photons_per_step_per_gpu": int(spec["n_photons"]),
            "sensors": [s["kind"] for s in spec["sensors"]], "layers": len(spec["layers"]),
            "max_events": spec.get("max_events", 1000), "precision": args.precision,
            "l2": "flushed between steps (256 MiB write)", "parallelism": f"photon-range x{n_gpus}",
            "seed": spec["seed"], "block_size": args.block_size or 256,
            "blocks_per_sm": args.blocks_per_sm or "auto",
            "batch_photons": args.batch_photons or (32 << 20),
            "cbs_history": "tracked per event" if args.no_replay else "replayed for CBS-grid hits",
            "amplitude_tables": "shared memory (bulk copies)" if args.stage_tables else "global via L1",
            "tally_mode": args.tally_mode}


# ------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), samples=len(sm))
        out["reasons"] = sorted(reasons)
        os.unlink(self.path)
        return out


# ------------------------------------------------------------------ reference (CPU)
def reference_module():
    from oracle import pyoracle as O
    lm = O.reference_module("perf")
    lm.set_log_level(lm.LogLevel.off)
    return lm


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_sample(spec, seconds, threads):
    """Time the reference's run_simulation_parallel on a bounded photon sample sized
    for about `seconds` of work; returns (photons/s, photons, wall)."""
    from luminis_mc_b200 import workloads as W
    lm = reference_module()

    def run(n, seed):
        cfg, _, keep = W.build(lm, spec, n_photons=n, seed=seed, n_threads=threads)
        cfg.pin_threads_to_cores = True
        t0 = time.perf_counter()
        lm.run_simulation_parallel(cfg)
        return time.perf_counter() - t0

    n = max(threads * 50, 2000)
    dt = run(n, 1)
    while dt < 1.0 and n < 10 ** 9:
        n *= 4
        dt = run(n, 2)
    n = max(n, int(n * seconds / dt))
    dt = run(n, 3)
    return n / dt, n, dt


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    spec = workload_spec(args.workload, args.photons)
    threads = os.cpu_count() or 1
    from luminis_mc_b200 import workloads as W
    lm = reference_module()
    # size one step to a bounded sample (~cpu_seconds of work)
    rate, n, _ = reference_sample(spec, args.cpu_seconds / 2, threads)
    n_step = max(1000, int(rate * args.cpu_seconds / 2))
    times = []
    for i in range(args.warmup + args.steps):
        cfg, _, keep = W.build(lm, spec, n_photons=n_step, seed=1000 + i, n_threads=threads)
        cfg.pin_threads_to_cores = True
        t0 = time.perf_counter()
        lm.run_simulation_parallel(cfg)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = n_step * len(times) / total
    line = {"metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded media of the workload)", "impl": "reference",
            "config": config_block(spec, args, 1) | {"photons_per_step_per_gpu": n_step,
                                                      "precision": "fp64"},
            "cpu_baseline": {"value": value, "unit": "photons/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{n_step} photons per step of {spec['name']}, "
                                       f"run_simulation_parallel with n_threads={threads}"},
            "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- ours
def run_ours(args):
    import numpy as np
    import torch

    import luminis_mc_b200 as lm
    from luminis_mc_b200 import _native as N
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    spec = workload_spec(args.workload, args.photons)
    P = int(spec["n_photons"])
    cfg, handles, keep = W.build(lm, spec)
    run = DeviceRun(cfg, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    seed = int(spec["seed"])
    base = rank * P                       # this rank's photon range, per step

    def step(k):
        flush.zero_()
        st, _ = run.run(P, seed, begin=(k * world * P) + base, precision=args.precision,
                        stream=stream.cuda_stream, block_size=args.block_size,
                        blocks_per_sm=args.blocks_per_sm, batch_photons=args.batch_photons,
                        stage_tables=args.stage_tables, no_replay=args.no_replay,
                        tally_mode=args.tally_mode)
        return st

    for k in range(args.warmup):
        step(k)
    barrier()
    stats = []
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            stats.append(step(args.warmup + k))
        barrier()
    clocks = clk.summary()
    kernel_ms = sum(s["kernel_ms"] for s in stats)
    t = torch.tensor([kernel_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    photons_all = P * world * args.steps
    value = photons_all / (total_ms * 1e-3)
    events = sum(s["events"] for s in stats)
    steps_ = sum(s["steps"] for s in stats)
    photons_done = sum(s["photons"] for s in stats)
    assert photons_done == P * args.steps, (photons_done, P * args.steps)

    # roofline: the transport kernel is FP32/SFU issue-bound; measured FMA peak.
    # achieved = algorithmic flops of its launches / their own CUDA-event time
    peak_tflops, _ = N.probe_fp32_peak(200000)
    transport_ms = sum(s["transport_ms"] for s in stats)
    transport_launches = sum(s["transport_launches"] for s in stats)
    achieved_tflops = events * FLOP_PER_EVENT / (transport_ms * 1e-3) / 1e12
    per_photon = TRAFFIC_BYTES_PER_PHOTON.get(spec["name"]) if args.precision == "fp32" else None
    traffic = per_photon * P / max(1, transport_launches // args.steps) if per_photon else None
    # one transport, one CBS replay (when the scene replays) and one tally kernel per batch
    launches = 2 * transport_launches + sum(s.get("replay_launches", 0) for s in stats)

    variants = {}
    if args.variant_steps > 0:
        variants = measure_variants(args, spec, local, stream, flush, world, rank, dist)

    # end-to-end through the public API: host tally arrays, copies inside
    e2e = None
    if not args.no_e2e:
        e2e_ms, e2e_device_ms = [], []
        cfg2, h2, keep2 = W.build(lm, spec)
        tally_bytes = run.transport.tally_size * 8
        table_bytes = 0
        for layer in cfg2.sample.layers:
            m = layer.medium
            table_bytes += m._s1.nbytes + m._s2.nbytes
            v, c = m.phase_function._table()
            if v is not None:
                table_bytes += 2 * v.nbytes
        # one untimed call first: the process's one-time costs (pinned read-back halves,
        # first touch of the sensors' host arrays) are not part of a step
        cfg2.seed = seed + 76
        lm.run_simulation_parallel(cfg2, precision=args.precision)
        for k in range(2):
            # every timed call uploads its scene's tables: the scene the public API keeps
            # between calls is released first (outside the timed region)
            lm.release_gpu_cache()
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            cfg2.seed = seed + 77 + k
            lm.run_simulation_parallel(cfg2, precision=args.precision)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            e2e_device_ms.append(lm.last_run_stats()["kernel_ms"])
        lm.release_gpu_cache()
        worst = torch.tensor([max(e2e_ms)], dtype=torch.float64, device=f"cuda:{local}")
        if dist is not None:
            dist.all_reduce(worst, op=dist.ReduceOp.MAX)
        e2e = {"value": P * world / (float(worst.item()) * 1e-3), "unit": "photons/s",
               "h2d_bytes_per_step": int(table_bytes),
               "d2h_bytes_per_step": int(tally_bytes + 256),
               "path": "luminis_mc_b200.run_simulation_parallel(config) with numpy tallies",
               "calls_ms": {"wall": [round(x, 2) for x in e2e_ms],
                            "device": [round(x, 2) for x in e2e_device_ms]}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            rate, n, dt = reference_sample(spec, args.cpu_seconds, threads)
            cpu = {"value": rate, "unit": "photons/s", "cores": threads, "kind": "reference",
                   "sample": f"{n} photons of {spec['name']} in {dt:.1f} s, reference "
                             f"run_simulation_parallel (oracle/_ref/perf) with n_threads={threads}",
                   "cpu_model": cpu_model()}
            rate1, n1, dt1 = reference_sample(spec, 3.0, 1)
            cpu["single_thread"] = {"value": rate1, "unit": "photons/s",
                                    "sample": f"{n1} photons in {dt1:.1f} s, n_threads=1"}
        except Exception as exc:          # the reference build is optional where the bench runs
            cpu = {"value": None, "unit": "photons/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "fp32" else "f64",
                "data": "synthetic (seeded media of the workload)",
                "config": config_block(spec, args, world),
                "events_per_s": events * world / (total_ms * 1e-3),
                "steps_per_s": steps_ * world / (total_ms * 1e-3),
                "events_per_photon": events / max(1, photons_done),
                "roofline": {"bound": "fp32-issue", "achieved": achieved_tflops,
                             "peak": peak_tflops, "unit": "TFLOP/s",
                             "frac": achieved_tflops / peak_tflops,
                             "peak_source": "measured: FFMA probe (lmc_probe_fp32_peak) on this GPU",
                             "flop_per_event": FLOP_PER_EVENT,
                             "kernel": "transport_kernel", "launches": transport_launches,
                             "ms_per_launch": transport_ms / max(1, transport_launches),
                             "traffic": traffic,
                             "traffic_source": "ncu dram bytes per photon x photons per launch"
                                               if traffic else None,
                             # the same launches against HBM: the hit queue is all they move
                             "hbm_view": ({"achieved": traffic / (transport_ms / max(1, transport_launches)) / 1e6,
                                           "peak": HBM_PEAK_GBS[0], "unit": "GB/s",
                                           "frac": traffic / (transport_ms / max(1, transport_launches)) / 1e6
                                           / HBM_PEAK_GBS[0], "peak_source": HBM_PEAK_GBS[1]}
                                          if traffic else None)},
                "replayed_per_photon": sum(s.get("replayed", 0) for s in stats) / max(1, photons_done),
                "arms": headline_arms(value, e2e, variants),
                "variants": variants,
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    run.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def headline_arms(value, e2e, variants):
    """The three arms of the headline metric side by side: binary32 transport (this
    line), binary64 throughout (the like-for-like arm of the reference's binary64 CPU
    path) and binary32 with likelihood-ratio derivatives; device photons/s and the
    end-to-end photons/s of each through its public API."""
    def arm(rec, workload):
        if not rec:
            return None
        return {"value": rec.get("value"), "e2e": (rec.get("e2e") or {}).get("value"),
                "unit": "photons/s", "workload": workload}
    return {"fp32": {"value": value, "e2e": (e2e or {}).get("value"), "unit": "photons/s",
                     "workload": "bilayer_rgd_mie"},
            "fp64": arm(variants.get("fp64"), "bilayer_rgd_mie"),
            "fp32_adjoint": arm(variants.get("fp32_adjoint"), "bilayer_hg (differentiable)")}


def measure_variants(args, spec, local, stream, flush, world, rank, dist):
    """The two other arms of the headline metric on this GPU: the same workload in
    FP64 throughout, and FP32 transport with the likelihood-ratio derivatives of the
    differentiable configuration (HG bilayer, 1e7 photons, radial fluence profile of
    100 bins to 5 mm, CBS cone); and the batched sweep of 256 Mie media in one launch
    (plain, replayed from a CUDA graph, and as one launch per medium).  photons/s from
    the device time of the runs.  `--variants` picks a subset."""
    import torch

    def max_ms(ms):
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    out = {}
    sel = set(args.variants.split(","))
    if "fp64" in sel:
        out.update(measure_fp64(args, spec, local, stream, flush, world, rank, max_ms))
    if "differentiable" in sel:
        out.update(measure_differentiable(args, local, stream, flush, world, rank, max_ms))
    if "sweep" in sel:
        out.update(measure_sweep(args, local, stream, flush, world, rank, max_ms))
    if "estimator" in sel:
        out.update(measure_estimator(args, local, stream, flush, world, rank, max_ms))
    if "f2" in sel:
        out.update(measure_f2(args, local, stream, flush, world, rank, max_ms))
    if "long_paths" in sel:
        out.update(measure_long_paths(args, local, stream, flush, world, rank, max_ms))
    return out


def measure_long_paths(args, local, stream, flush, world, rank, max_ms):
    """The precision-stress workload (mie_long_paths: mu_s = 100/mm, mu_a = 1e-4/mm,
    ~1.1e4 events per photon, FarFieldCBS 400 bins to 20 mrad, 256 x 256 speckle grid),
    linear and circular polarisation, binary32 and binary64 transport, 1e7 photons per
    run.  photons/s and scattering events/s from device time.  5.5e-3 of the photons reach
    MAX_EVENTS (1e6 events) and carry half of all events; a run ends with the last of them
    running on a nearly idle GPU, one event after another, for a few seconds: at 2e6
    photons that tail is most of the run (~0.32 M photons/s in either precision), at 1e7
    the bulk of the work hides most of it."""
    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    out = {}
    P = 10_000_000
    for circ in (False, True):
        spec = W.mie_long_paths(P, 12345, circular=circ)
        cfg, _, keep = W.build(lm, spec)
        rec = {"workload": spec["name"], "photons": P, "unit": "photons/s"}
        for key, prec in (("fp32", "fp32"), ("fp64", "fp64")):
            run = DeviceRun(cfg, device=f"cuda:{local}")
            run.run(20_000, 7, precision=prec, stream=stream.cuda_stream, max_events=1000)  # warm-up
            flush.zero_()
            st, _ = run.run(P, 12345, begin=(1 + rank) * P, precision=prec, stream=stream.cuda_stream)
            run.close()
            ms = max_ms(st["kernel_ms"])
            rec[key] = {"value": P * world / (ms * 1e-3), "events_per_s": st["events"] * world / (ms * 1e-3),
                        "events_per_photon": st["events"] / P, "photons_at_max_events": st["cap"]}
        out[f"long_paths_{'circular' if circ else 'linear'}"] = rec
    return out


def f2_specs(n_photons):
    """The transport's optional parts on the headline geometry: a three-species
    MixtureLayer slab, the Absorption recorder on a 100 x 100 (r, z) grid, and a
    StatisticsSensor with event, theta, phi and depth histograms beside the sensors."""
    from luminis_mc_b200 import workloads as W
    mix = W.mixture_bilayer(n_photons, 12345)
    absorb = W.bilayer_rgd_mie(n_photons, 12345)
    absorb["name"] = "bilayer_rgd_mie_absorption"
    absorb["absorption"] = {"radius": 5.0, "depth": 2.0, "d_r": 0.05, "d_z": 0.02}
    stats = W.bilayer_rgd_mie(n_photons, 12345)
    stats["name"] = "bilayer_rgd_mie_statistics"
    stats["sensors"].append({"kind": "statistics", "z": 0.0, "absorb": False, "events": 200,
                             "theta": [0.0, 3.1416, 90], "phi": [0.0, 6.2832, 36],
                             "depth": [2.0, 100]})
    return {"mixture_bilayer": mix, "absorption": absorb, "statistics": stats}


def measure_f2(args, local, stream, flush, world, rank, max_ms):
    """MixtureLayer, Absorption recorder and StatisticsSensor workloads (FP32, device time),
    each beside the reference's own run_simulation_parallel on this host's cores."""
    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    out = {}
    P = 10_000_000
    for key, spec in f2_specs(P).items():
        cfg, _, keep = W.build(lm, spec)
        run = DeviceRun(cfg, device=f"cuda:{local}")
        run.run(P // 10, 99, precision="fp32", stream=stream.cuda_stream)
        flush.zero_()
        st, _ = run.run(P, 12345, begin=(1 + rank) * P, precision="fp32", stream=stream.cuda_stream)
        run.close()
        ms = max_ms(st["kernel_ms"])
        rec = {"value": P * world / (ms * 1e-3), "unit": "photons/s", "workload": spec["name"],
               "photons": P, "events_per_photon": st["events"] / P}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                rate, n, dt = reference_sample(spec, 3.0, os.cpu_count() or 1)
                rec["cpu_reference"] = {"value": rate, "unit": "photons/s", "cores": os.cpu_count(),
                                        "sample": f"{n} photons in {dt:.1f} s, reference "
                                                  f"run_simulation_parallel (oracle/_ref/perf)"}
            except Exception as exc:
                rec["cpu_reference"] = {"value": None, "sample": f"unavailable: {exc}"}
        out[f"f2_{key}"] = rec
    return out


def measure_fp64(args, spec, local, stream, flush, world, rank, max_ms):
    """FP64 throughout on the headline workload, device time and end to end."""
    import torch

    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    P = int(spec["n_photons"])
    cfg, _, keep = W.build(lm, spec)
    run = DeviceRun(cfg, device=f"cuda:{local}")
    ms = 0.0
    for k in range(1 + args.variant_steps):
        flush.zero_()
        st, _ = run.run(P, int(spec["seed"]), begin=(k * world + rank) * P, precision="fp64",
                        stream=stream.cuda_stream)
        if k >= 1:
            ms += st["kernel_ms"]
    run.close()
    ms = max_ms(ms)
    rec = {"value": P * world * args.variant_steps / (ms * 1e-3), "unit": "photons/s",
           "workload": spec["name"], "steps": args.variant_steps}
    if not args.no_e2e:
        # end to end through the public API in FP64: the like-for-like arm of the
        # reference's all-binary64 CPU path
        cfg2, _, keep2 = W.build(lm, spec)
        cfg2.seed = int(spec["seed"]) + 90
        lm.run_simulation_parallel(cfg2, precision="fp64")          # untimed first call
        wall = []
        for k in range(2):
            lm.release_gpu_cache()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            cfg2.seed = int(spec["seed"]) + 91 + k
            lm.run_simulation_parallel(cfg2, precision="fp64")
            torch.cuda.synchronize()
            wall.append((time.perf_counter() - t0) * 1e3)
        lm.release_gpu_cache()
        worst = max_ms(max(wall))
        rec["e2e"] = {"value": P * world / (worst * 1e-3), "unit": "photons/s",
                      "path": "luminis_mc_b200.run_simulation_parallel(config, precision='fp64') "
                              "with numpy tallies",
                      "calls_ms": [round(x, 2) for x in wall]}
    return {"fp64": rec}


def measure_differentiable(args, local, stream, flush, world, rank, max_ms):
    """FP32 on the differentiable workload, without and with the likelihood-ratio
    derivatives (HG bilayer, 1e7 photons, radial fluence profile, CBS cone)."""
    import numpy as np
    import torch

    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.adjoint import AdjointTransport
    from luminis_mc_b200.device import DeviceRun

    out = {}

    aspec = W.bilayer_hg(10_000_000, 2024)
    acfg, _, akeep = W.build(lm, aspec)
    PA = int(aspec["n_photons"])
    run = DeviceRun(acfg, device=f"cuda:{local}")
    ms = 0.0
    for k in range(1 + args.variant_steps):
        flush.zero_()
        st, _ = run.run(PA, 2024, begin=(k * world + rank) * PA, precision="fp32",
                        stream=stream.cuda_stream)
        if k >= 1:
            ms += st["kernel_ms"]
    run.close()
    ms = max_ms(ms)
    out["fp32_differentiable_workload"] = {
        "value": PA * world * args.variant_steps / (ms * 1e-3), "unit": "photons/s",
        "workload": "bilayer_hg (differentiable), no derivatives", "steps": args.variant_steps}
    tr = AdjointTransport(acfg, radial_sensor=1, radial_bins=100, radial_max=5.0,
                          device=f"cuda:{local}")
    ms = 0.0
    for k in range(1 + args.variant_steps):
        flush.zero_()
        _, _, st = tr.run(PA, 2024, precision="fp32", begin=(k * world + rank) * PA,
                          stream=stream.cuda_stream)
        if k >= 1:
            ms += st["kernel_ms"]
    ms = max_ms(ms)
    out["fp32_adjoint"] = {"value": PA * world * args.variant_steps / (ms * 1e-3),
                           "unit": "photons/s", "workload": "bilayer_hg (differentiable)",
                           "parameters": 8, "outputs": "total + 100 radial bins + CBS S0 cone",
                           "steps": args.variant_steps}
    if not args.no_e2e:
        # end to end through the autograd function: parameters from a host tensor (scene
        # tables re-uploaded), forward on the GPU, outputs to the host, backward
        # (J^T g on the GPU) and the gradient to the host
        from luminis_mc_b200.adjoint import lr_transport
        wall = []
        for k in range(3):
            theta = torch.tensor(tr.parameters(), dtype=torch.float64, requires_grad=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            y = lr_transport(theta, tr, PA, 2024 + 31 * k, precision="fp32")
            y.sum().backward()
            g = theta.grad.numpy().copy()
            wall.append((time.perf_counter() - t0) * 1e3)
        worst = max_ms(max(wall[1:]))           # the first call is untimed
        out["fp32_adjoint"]["e2e"] = {
            "value": PA * world / (worst * 1e-3), "unit": "photons/s",
            "path": "luminis_mc_b200.adjoint.lr_transport(theta) forward + backward, host tensors",
            "calls_ms": [round(x, 2) for x in wall[1:]], "grad_finite": bool(np.isfinite(g).all())}
    tr.close()

    return out


def measure_sweep(args, local, stream, flush, world, rank, max_ms):
    """The batched sweep: 256 single-layer Mie media (seeded radius, mu_s, mu_a, photon
    counts log-uniform 1e5..1e7) in one launch, against one launch per medium; with and
    without each medium's gradients; launch shape from the autotuner."""
    import numpy as np
    import torch

    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.adjoint import AdjointTransport

    out = {}
    from luminis_mc_b200 import _native as N
    from luminis_mc_b200.sweep import SweepRun
    from luminis_mc_b200.simulation import Transport
    _, _, _, counts = W.mie_sweep_parameters()
    sspecs = [W.mie_sweep(i, seed=2026) for i in range(len(counts))]
    # set-up tables of the 256 species: one at a time on the host (the constructors),
    # against one lmc_mie_tables batch on the GPU (same numbers bit for bit)
    particles = [(sp["phases"][0]["wavelength"], sp["phases"][0]["radius"],
                  sp["phases"][0]["n_particle"], sp["phases"][0]["n_medium"]) for sp in sspecs]
    host_s, gpu_s, split = [], [], []
    for _ in range(3):
        t0 = time.perf_counter()
        for q in particles:
            lm.MieMedium(lm.MiePhaseFunction(*q, 1000, 0.0, math.pi), q[1], q[2], q[3], q[0])
        host_s.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        split.append({})
        lm.mie_species(particles, 1000, 0.0, math.pi, timing=split[-1])
        gpu_s.append(time.perf_counter() - t0)
    scfgs = W.build_mie_sweep(lm, sspecs)
    sw = SweepRun(scfgs, device=f"cuda:{local}")
    sw.set_photons(counts)
    total = int(counts.sum())
    tuned = sw.autotune(2025 + rank * 7919, precision="fp32", sample_photons=20_000_000)
    sw.run(2026 + rank * 7919, precision="fp32", stream=stream.cuda_stream)   # grows the queue
    flush.zero_()
    st = sw.run(2027 + rank * 7919, precision="fp32", stream=stream.cuda_stream)
    sweep_ms = max_ms(st["kernel_ms"])
    g = sw.capture(2028 + rank * 7919, precision="fp32")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    e0.record(stream)
    g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    graph_ms = max_ms(e0.elapsed_time(e1))
    del g
    # the same sweep with each medium's CBS S0 grids and their derivatives with respect
    # to its (mu_a, mu_s, mean free path, g): one launch, against one adjoint launch
    # per medium (sum of their device times)
    sw.run_adjoint(2029 + rank * 7919, precision="fp32", stream=stream.cuda_stream)
    flush.zero_()
    _, st = sw.run_adjoint(2030 + rank * 7919, precision="fp32", stream=stream.cuda_stream)
    sweep_adj_ms = max_ms(st["kernel_ms"])
    sw.close()
    seq_adj_ms = 0.0
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]])
    for c, n, o in zip(scfgs, counts, offs):
        tr = AdjointTransport(c, device=f"cuda:{local}")
        _, _, st = tr.run(int(n), 2030 + rank * 7919, precision="fp32", begin=int(o),
                          stream=stream.cuda_stream)
        seq_adj_ms += st["kernel_ms"]
        tr.close()
    seq_adj_ms = max_ms(seq_adj_ms)
    trs = [Transport(c) for c in scfgs]
    bufs = [torch.zeros(max(t.tally_size, 1), dtype=torch.float64, device=f"cuda:{local}")
            for t in trs]
    # one launch per medium: every medium's run once (queues allocated), then timed
    # back to back on a stream of their own, and as the sum of each run's device time
    side = torch.cuda.Stream(device=f"cuda:{local}")
    for t, b, n, o in zip(trs, bufs, counts, offs):
        t.run_device(b.data_ptr(), int(n), 2026 + rank * 7919, int(o), want_stats=False,
                     precision="fp32", stream=side.cuda_stream)
    flush.zero_()
    torch.cuda.synchronize()
    e0.record(side)
    for t, b, n, o in zip(trs, bufs, counts, offs):
        t.run_device(b.data_ptr(), int(n), 2027 + rank * 7919, int(o), want_stats=False,
                     precision="fp32", stream=side.cuda_stream)
    e1.record(side)
    torch.cuda.synchronize()
    seq_ms = max_ms(e0.elapsed_time(e1))
    seq_dev_ms = 0.0
    for t, b, n, o in zip(trs, bufs, counts, offs):
        seq_dev_ms += t.run_device(b.data_ptr(), int(n), 2027 + rank * 7919, int(o),
                                   want_stats=True, precision="fp32",
                                   stream=side.cuda_stream)["kernel_ms"]
    seq_dev_ms = max_ms(seq_dev_ms)
    for t in trs:
        t.close()
    out["sweep_256_media"] = {
        "value": total * world / (sweep_ms * 1e-3), "unit": "photons/s", "precision": "fp32",
        "photons": total, "media": len(counts), "graph_replay": total * world / (graph_ms * 1e-3),
        "sequential_launches": total * world / (seq_ms * 1e-3),
        "sequential_device_time": total * world / (seq_dev_ms * 1e-3),
        "with_gradients": total * world / (sweep_adj_ms * 1e-3),
        "with_gradients_sequential_device_time": total * world / (seq_adj_ms * 1e-3),
        "gradients": "CBS S0 coherent + incoherent grids and d/d(mu_a, mu_s, mfp, g) per medium",
        "launch_shape": {"picked_by": "lmc_autotune on a 2e7-photon scaled copy of the sweep",
                         **{k: tuned[k] for k in ("block_size", "blocks_per_sm", "batch_photons",
                                                  "n_tried")},
                         "tally_mode": {v: k for k, v in N.TALLY_MODES.items()}.get(
                             tuned["tally_mode"], tuned["tally_mode"])},
        "workload": "256 single-layer Mie media, FarFieldCBS 100x1 each, seeded draws "
                    "(numpy default_rng(2026))",
        "tables": {"species": len(particles), "host_s": round(sorted(host_s)[1], 4),
                   "gpu_s": round(sorted(gpu_s)[1], 4),
                   "gpu_split_ms": {k: round(sorted(t[k] for t in split)[1], 3) for k in split[0]},
                   "what": "MiePhaseFunction (1001-node CDF) + MieMedium (1000-node S1/S2) "
                           "per species; host: the constructors one species at a time on one "
                           "thread; gpu: lmc_mie_tables, host coefficients + device sums, "
                           "wall time including copies (median of 3)"}}

    return out


def measure_estimator(args, local, stream, flush, world, rank, max_ms):
    """Estimator-mode FarFieldCBS (the reference's last-flight CBS estimate at every
    vertex), mie_cbs_small geometry with its 100-bin grid, against the reference's own
    estimator on this host's cores."""
    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    out = {}
    espec = W.mie_cbs_small(args.estimator_photons, 4242)
    espec["sensors"] = [dict(espec["sensors"][0], estimator=True)]
    ecfg, _, ekeep = W.build(lm, espec)
    PE = int(espec["n_photons"])
    from luminis_mc_b200 import _native as N
    n_bins = int(round(espec["sensors"][0]["theta_max"] / espec["sensors"][0]["d_theta"]))
    for prec in ("fp64", "fp32"):
        run = DeviceRun(ecfg, device=f"cuda:{local}")
        run.run(20_000, 4242, precision=prec, stream=stream.cuda_stream)
        flush.zero_()
        st, _ = run.run(PE, 4242, begin=(1 + rank) * PE, precision=prec, stream=stream.cuda_stream)
        run.close()
        ms = max_ms(st["kernel_ms"])
        out[f"estimator_{prec}"] = {"value": PE * world / (ms * 1e-3), "unit": "photons/s",
                                    "workload": "mie_cbs_small, FarFieldCBS 100x1 in estimator mode",
                                    "photons": PE}
        if prec == "fp32":
            # every estimated vertex (the sensor's hit count) against every bin of the grid
            pairs = st["hits"][0] * n_bins
            peak, _ = N.probe_fp32_peak(200000)
            achieved = pairs * FLOP_PER_EST_PAIR / (st["transport_ms"] * 1e-3) / 1e12
            out["estimator_fp32"]["roofline"] = {
                "bound": "fp32-issue", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "flop_per_pair": FLOP_PER_EST_PAIR, "pairs": pairs,
                "kernel": "transport_kernel (estimator mode)", "ms": st["transport_ms"],
                "peak_source": "measured: FFMA probe (lmc_probe_fp32_peak) on this GPU"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, n, dt = reference_sample(espec, 6.0, os.cpu_count() or 1)
            out["estimator_fp64"]["cpu_reference"] = {
                "value": rate, "unit": "photons/s", "cores": os.cpu_count(),
                "sample": f"{n} photons in {dt:.1f} s, reference run_simulation_parallel "
                          f"(oracle/_ref/perf), estimator mode"}
        except Exception as exc:
            out["estimator_fp64"]["cpu_reference"] = {"value": None, "sample": f"unavailable: {exc}"}
    return out


def precision_report(args):
    """Per sensor: FP32 transport (u24 stream), with the CBS phase in binary64 and in
    binary32, against FP64 transport on the same u24 numbers (stream_format=1), i.e.
    precision error alone, next to the Monte Carlo noise of the same tally (FP64 on two
    independent seeds).  The long-path workloads run --photons photons (1e7 by
    default).  One JSON line per workload."""
    import numpy as np
    import torch

    import luminis_mc_b200 as lm
    from luminis_mc_b200 import workloads as W
    from luminis_mc_b200.device import DeviceRun

    torch.cuda.set_device(0)
    n3 = args.photons or 10_000_000
    cases = [("mie_cbs_small", W.mie_cbs_small(1_000_000, 12345)),
             ("bilayer_rgd_mie", W.bilayer_rgd_mie(10_000_000, 12345)),
             ("mie_long_paths_linear", W.mie_long_paths(n3, 12345)),
             ("mie_long_paths_circular", W.mie_long_paths(n3, 12345, circular=True))]
    # arms: binary32 transport with the CBS phase in binary64 (the default) and in
    # binary32; binary64 on the same u24 numbers (the oracle of both); binary64 on another
    # seed (the Monte Carlo noise of the same tally)
    arms = (("fp32", "fp32", 0, 0, "fp64"), ("fp32_phase32", "fp32", 0, 0, "fp32"),
            ("fp64", "fp64", 1, 0, "fp64"), ("fp64_other_seed", "fp64", 1, 1, "fp64"))
    for name, spec in cases:
        cfg, _, keep = W.build(lm, spec)
        n, seed = int(spec["n_photons"]), int(spec["seed"])
        res = {}
        for key, prec, fmt, dseed, phase in arms:
            run = DeviceRun(cfg)
            st, _ = run.run(n, seed + dseed, precision=prec, stream_format=fmt, cbs_phase=phase,
                            max_events=spec["max_events"])
            res[key] = ([t.copy() for t in run.host_tallies()], st, st["kernel_ms"])
            run.close()
        sensors = []
        for i, s in enumerate(spec["sensors"]):
            b, c = res["fp64"][0][i], res["fp64_other_seed"][0][i]
            comps = []
            for q in range(b.shape[0]):
                bq = b[q].ravel()
                scale = float(np.abs(bq).max()) or 1.0
                l2 = float(np.linalg.norm(bq)) or 1.0
                comp = {"rel_l2_mc_noise": float(np.linalg.norm(c[q].ravel() - bq)) / l2}
                for key in ("fp32", "fp32_phase32"):
                    aq = res[key][0][i][q].ravel()
                    comp[key] = {"max_abs_err_of_max": float(np.abs(aq - bq).max()) / scale,
                                 "rel_l2_err": float(np.linalg.norm(aq - bq)) / l2,
                                 "total_rel_err": float(abs(aq.sum() - bq.sum()) / (abs(bq.sum()) or 1.0))}
                comps.append(comp)
            sensors.append({"sensor": s["kind"], "components": comps})
        line = {"workload": name, "photons": n, "seed": seed,
                "events": {k: res[k][1]["events"] for k in res},
                "hits": {k: res[k][1]["hits"][:len(spec["sensors"])] for k in res},
                "photons_per_s": {k: n / (res[k][2] * 1e-3) for k in res},
                "sensors": sensors}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.precision_report:
        precision_report(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
