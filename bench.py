#!/usr/bin/env python
"""Headline benchmark: the P3BCA Simulation step on one B200 (C3: N=131072 uniform particles at
density 2.048 in a 40^3 box, cutoff 2, mass 1, zero velocity, dt 0.001, g = (0,-9.81,0)), mixed
precision, with the FP64 drop-in measured beside it.  Metric: triplets/s (triplets inside the
cutoff evaluated per second, the count Simulation::GetNumParticleInteractions returns) and
ms/step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c3|c3c15|c2|c1|c4] [--precision mixed|fp64]

One process per GPU (torchrun for N > 1).  The path does not shard (one GPU holds the whole cell
grid), so N GPUs run N independent replicas ("scaling": "weak"); no collective is on the data
path, the only NCCL calls are the barrier and the max-over-ranks of the timed region.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events on the stream the
library runs on (torch's current stream, handed to the context), with a 256 MiB write between
steps to flush L2 (the working set is smaller than L2).  `value` = all ranks' triplets / max over
ranks of the summed step times.  `e2e` repeats the step through the C ABI with the particle state
copied in from pinned host memory and back out every step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "c3": dict(desc="P3BCA, N=131072 uniform at density 2.048 (box 40^3), cutoff 2, 1 step/iteration",
               algorithm="p3bca", n=131072, cutoff=2.0, gen="uniform"),
    "c3c15": dict(desc="P3BCA, N=131072 uniform at density 2.048 (box 40^3), cutoff 1.5",
                  algorithm="p3bca", n=131072, cutoff=1.5, gen="uniform"),
    "c2": dict(desc="AUTA, N=8192 uniform in 20^3, no cutoff", algorithm="auta", n=8192, cutoff=0.0, gen="uniform",
               box=20.0),
    "c2nata": dict(desc="NATA, N=8192 uniform in 20^3, no cutoff", algorithm="nata", n=8192, cutoff=0.0,
                   gen="uniform", box=20.0),
    "c1": dict(desc="AUTA, N=512 uniform in 10^3, no cutoff", algorithm="auta", n=512, cutoff=0.0, gen="uniform",
               box=10.0),
    "c4": dict(desc="P3BCA, N=262144 clustered Gaussian (256 clusters, sigma 1) in 64^3, cutoff 2",
               algorithm="p3bca", n=262144, cutoff=2.0, gen="clustered", box=64.0),
    "c5": dict(desc="64 systems, N uniform in 512..4096 at density 2.048, batched AUTA and P3BCA (cutoff 2), "
                    "forward and adjoint", algorithm="batch", n=0, cutoff=2.0, gen="batch"),
}
FLOP_PER_TRIPLET = 120  # the fixed, formulation-independent credit per triplet inside the cutoff
DT, G = 0.001, (0.0, -9.81, 0.0)


def make_input(w, device=None):
    """The workload's particles: the reference generator's sequence after its 6-digit CSV round trip.
    With a device, generated on the GPU (tbmd_generate_particles) and read back; otherwise by the
    host generator (the reference arm's path)."""
    from threebodymdalgorithms_b200 import generators as gen
    side = w.get("box") or gen.box_for_density(w["n"], 2.048)
    if device is not None:
        from threebodymdalgorithms_b200 import Context
        ctx = Context("auta", device=device)
        if w["gen"] == "uniform":
            ctx.generate(kind="uniform", n=w["n"], box=(side, side, side))
        else:
            ctx.generate(kind="clusteredgauss", n=w["n"], n_clusters=256, box=(side, side, side))
        st = ctx.get_state()
        ctx.close()
        return {k: st[k] for k in ("id", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")}
    if w["gen"] == "uniform":
        return gen.as_csv_values(gen.uniform(w["n"], (side, side, side), 1.0))
    return gen.as_csv_values(gen.clustered_gauss(w["n"], 256, (side,) * 3, 0.0, 1.0, 1.0))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the first sample arrives after nvidia-smi has started; wait for it (at most 5 s) so
            # that the samples cover the timed region
            t0 = time.monotonic()
            while not self.lines and time.monotonic() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def _all_reduce(v, world, op):
    """v reduced over all ranks (NCCL: on the GPU; gloo: on the CPU)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allreduce_max(v, world):
    import torch.distributed as dist
    return _all_reduce(v, world, dist.ReduceOp.MAX)


def allreduce_sum(v, world):
    import torch.distributed as dist
    return _all_reduce(v, world, dist.ReduceOp.SUM)


def aggregate(triplets_rank, ms_rank, world):
    """Replicas: the whole job's triplets (sum over ranks) and its time (the slowest rank)."""
    return allreduce_sum(float(triplets_rank), world), allreduce_max(float(ms_rank), world)


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


# Algorithmic bytes per particle of the P3BCA step's cell build (predictor fused in), each array
# access counted once: k_predict_assign reads x, y, z, vx, vy, vz, ax (56 B), writes x, y, z (24 B),
# the cell index and the rank in the cell (8 B), and adds to the cell's count (8 B);
# k_scatter_gather reads the cell index, the rank and the cell's start (12 B) and x, y, z (24 B),
# and writes the sorted index and the slot (8 B), the sorted FP64 positions (24 B) and their FP32
# hi/lo copies (32 B).  The scan over the cells adds under 1 B per particle.
CELL_BUILD_BYTES = 96 + 100


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth in MEASURED_PEAKS.json, else the pool's fallback."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def cell_build_roofline(phase, n):
    ms = phase["ms"] / max(phase["calls"], 1)
    peak, src = hbm_peak()
    gbs = CELL_BUILD_BYTES * n / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    return {"bound": "hbm", "kernels": "k_predict_assign, k_cell_scan, k_scatter_gather", "ms": round(ms, 5),
            "bytes_per_particle": CELL_BUILD_BYTES, "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
            "frac": round(gbs / peak, 4), "peak_source": src}


def timed_steps(ctx, steps, flush, torch, reset=None):
    """Per-step CUDA-event times (ms) on the context's stream.  Before each step (untimed) the
    workload's input state is restored, so every step is the same step of the same input, and L2
    is flushed."""
    stream = torch.cuda.current_stream()
    times, counts, launches = [], [], 0
    for _ in range(steps):
        if reset is not None:
            reset()
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = ctx.kernel_launches()
        e0.record(stream)
        c = ctx.step(1)
        e1.record(stream)
        launches += ctx.kernel_launches() - l0
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        counts.append(int(c[0]))
    return times, counts, launches


def run_ours(args, world, rank, local):
    import torch
    from threebodymdalgorithms_b200 import Context
    from threebodymdalgorithms_b200._lib import load

    w = WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    # a dedicated stream: the library, the CUDA events and the L2 flush all run on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    st = make_input(w, device=local)
    n = len(st["x"])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def new_ctx(prec, graph=True):
        c = Context(w["algorithm"], prec, w["cutoff"], DT, G, 1.0, device=local, use_graph=graph,
                    stream=C.c_void_p(stream.cuda_stream))
        c.set_state(st)
        return c

    result = {}
    for prec in ([args.precision] + (["fp64"] if args.precision != "fp64" and not args.no_fp64 else [])):
        ctx = new_ctx(prec)
        reset = (lambda c=ctx: c.set_state(st))
        if not args.no_autotune:
            ctx.autotune(None)  # the project's autotuner picks the launch shape (untimed, no cache file)
        timed_steps(ctx, args.warmup, flush, torch, reset)
        barrier(world)
        with ClockSampler(local) as clk:
            times, counts, launches = timed_steps(ctx, args.steps, flush, torch, reset)
        barrier(world)
        trip_all, total_ms = aggregate(sum(counts), sum(times), world)
        result[prec] = dict(times=times, counts=counts, total_ms=total_ms, trip_all=trip_all, launches=launches,
                            clocks=clk.summary(), tuning=ctx.tuning())
        # per-phase device times of the same steps (eager mode, events between phases)
        ctx.set_profiling(True)
        timed_steps(ctx, min(args.steps, 10), flush, torch, reset)
        result[prec]["phases"] = ctx.phase_times()
        ctx.close()

    main = result[args.precision]
    trip_rank = float(sum(main["counts"]))
    trip_all = main["trip_all"]
    value = trip_all / (main["total_ms"] * 1e-3)
    ms_per_step = main["total_ms"] / args.steps

    # roofline of the dominant kernel (triplet forces), measured from the profiled pass
    ph = main["phases"]["triplets"]
    kern_ms = ph["ms"] / max(ph["calls"], 1)
    mean_trip = trip_rank / args.steps
    lib = load()
    lib.tbmd_probe_fma_tflops.restype = C.c_double
    lib.tbmd_probe_fma_tflops.argtypes = [C.c_int32, C.c_int32]
    fp32_peak = lib.tbmd_probe_fma_tflops(local, 0)
    fp64_peak = lib.tbmd_probe_fma_tflops(local, 1)
    peak = fp32_peak if args.precision == "mixed" else fp64_peak
    achieved = mean_trip * FLOP_PER_TRIPLET / (kern_ms * 1e-3) / 1e12
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get(f"{args.workload}:{args.precision}")
        except (ValueError, OSError):
            traffic = None
    roofline = {"bound": "fp32" if args.precision == "mixed" else "fp64", "achieved": round(achieved, 3),
                "peak": round(peak, 3), "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if peak > 0 else None,
                "traffic": traffic, "kernel": "k_p3bca" if w["algorithm"] == "p3bca" else f"k_{w['algorithm']}",
                "kernel_ms": round(kern_ms, 5), "flop_per_triplet": FLOP_PER_TRIPLET,
                "peak_source": "measured on this GPU by tbmd_probe_fma_tflops (FMA = 2 FLOP)",
                "phases_ms_per_step": {k: round(v["ms"] / max(v["calls"], 1), 5) for k, v in main["phases"].items()}}
    if w["algorithm"] == "p3bca" and w["cutoff"] > 0:
        roofline["cell_build"] = cell_build_roofline(main["phases"]["cells"], n)

    # end to end through the C ABI with host buffers (pinned), per step: state in, step, state out
    e2e = None
    if not args.no_e2e:
        ctx = new_ctx(args.precision)
        # one pinned SoA block per direction, a row per field (the library copies back-to-back fields
        # in one transfer)
        in_keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
        out_keys = in_keys + ("fx", "fy", "fz")
        in_block = torch.empty((len(in_keys), n), dtype=torch.float64).pin_memory().numpy()
        out_block = torch.empty((len(out_keys), n), dtype=torch.float64).pin_memory().numpy()
        pinned = {k: in_block[r] for r, k in enumerate(in_keys)}
        for k in in_keys:
            pinned[k][:] = st[k]
        ids = torch.from_numpy(np.asarray(st["id"], dtype=np.int32)).pin_memory().numpy()
        outs = {k: out_block[r] for r, k in enumerate(out_keys)}
        out_ids = torch.empty(n, dtype=torch.int32).pin_memory().numpy()
        from threebodymdalgorithms_b200._lib import dptr
        lib = ctx._lib

        IN = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
        OUT = IN + ("fx", "fy", "fz")
        ip = C.POINTER(C.c_int32)
        cnt = np.zeros(1, dtype=np.uint64)

        def e2e_fused():
            # tbmd_step_host: load, step, read back in one call, the copies overlapping the step
            ctx._check(lib.tbmd_step_host(ctx.handle, n, ids.ctypes.data_as(ip), *[dptr(pinned[k]) for k in IN], 1,
                                          cnt.ctypes.data_as(C.POINTER(C.c_uint64)), out_ids.ctypes.data_as(ip),
                                          *[dptr(outs[k]) for k in OUT]))
            return int(cnt[0])

        KSTEPS = 10
        cnt_k = np.zeros(KSTEPS, dtype=np.uint64)

        def e2e_ksteps():
            # the same call with K steps: the copies are paid once per K steps
            ctx._check(lib.tbmd_step_host(ctx.handle, n, ids.ctypes.data_as(ip), *[dptr(pinned[k]) for k in IN],
                                          KSTEPS, cnt_k.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          out_ids.ctypes.data_as(ip), *[dptr(outs[k]) for k in OUT]))
            return int(cnt_k.sum())

        def e2e_separate():
            ctx._check(lib.tbmd_set_particles(ctx.handle, n, ids.ctypes.data_as(ip), *[dptr(pinned[k]) for k in IN]))
            c = ctx.step(1)
            ctx._check(lib.tbmd_get_particles(ctx.handle, out_ids.ctypes.data_as(ip), *[dptr(outs[k]) for k in OUT]))
            return int(c[0])

        def e2e_time(fn):
            for _ in range(args.warmup):
                fn()
            barrier(world)
            ms, trips = [], 0
            for _ in range(args.steps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                trips += fn()
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            barrier(world)
            return allreduce_max(sum(ms), world), allreduce_sum(float(trips), world)

        tot, e2e_all = e2e_time(e2e_fused)
        tot_sep, _ = e2e_time(e2e_separate)
        ksteps = max(1, min(args.steps, 10))
        saved_steps, args.steps = args.steps, ksteps
        tot_k, trip_k = e2e_time(e2e_ksteps)
        args.steps = saved_steps
        # the device copies of one tbmd_step_host call: in, x y z vx vy vz ax m (ay and az, which no step
        # reads, stay on the host, where they are checked); out, x..az and fx fy fz (masses and IDs are
        # copied on the host)
        h2d, d2h = 8 * 8 * n, 12 * 8 * n
        e2e = {"value": e2e_all / (tot * 1e-3), "unit": "triplets/s", "ms_per_step": tot / args.steps,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "path": "tbmd_step_host (state in, step, state out in one C-ABI call), pinned host SoA blocks",
               "separate_calls_ms_per_step": tot_sep / args.steps,
               "k_steps": {"k": KSTEPS, "calls": ksteps, "ms_per_step": tot_k / (ksteps * KSTEPS),
                           "value": trip_k / (tot_k * 1e-3), "unit": "triplets/s",
                           "h2d_bytes_per_call": h2d, "d2h_bytes_per_call": d2h,
                           "path": "tbmd_step_host with K steps per call (state in, K steps, state out)"}}
        ctx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, st)

    if rank == 0:
        fp64 = result.get("fp64")
        line = {
            "metric": "triplets/s", "value": value, "unit": "triplets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 geometry + f64 accumulation" if args.precision == "mixed" else "f64",
            "data": "synthetic: the reference's particlegenerator sequences (mt19937 seed 926762934) after its 6-digit "
                    "CSV round trip, generated on the device; every timed step restarts from this input",
            "config": {"workload": f"{args.workload}: {w['desc']}", "algorithm": w["algorithm"], "n": n,
                       "cutoff": w["cutoff"], "precision": args.precision, "dt": DT, "g": list(G),
                       "triplets_per_step": mean_trip, "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"replicas x{world}", "graph": True, "tuning": main["tuning"]},
            "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": main["launches"],
            "clocks": main["clocks"],
        }
        if fp64 and args.precision != "fp64":
            f_ms = fp64["total_ms"] / args.steps
            line["fp64"] = {"ms_per_step": f_ms, "value": fp64["trip_all"] / (fp64["total_ms"] * 1e-3),
                            "triplets_per_step": float(np.mean(fp64["counts"])),
                            "phases_ms_per_step": {k: round(v["ms"] / max(v["calls"], 1), 5)
                                                   for k, v in fp64["phases"].items()},
                            "fp64_peak_tflops": round(fp64_peak, 3)}
            line["speedup_mixed_vs_fp64"] = f_ms / ms_per_step
            line["counts_equal_fp64_vs_mixed"] = fp64["counts"] == main["counts"]
        print(json.dumps(line), flush=True)


def run_trajectory(args, local):
    """A multi-step run of the workload (one tbmd_step(K) call: the step replayed K times from its
    CUDA graph), mixed and FP64 side by side: ms/step, triplets/s, per-step counts, and the AT
    potential, kinetic and gravitational energies at step 0 and step K, with the mixed run's
    difference from the FP64 run."""
    import torch
    from threebodymdalgorithms_b200 import Context

    w = WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    st = make_input(w, device=local)
    n = len(st["x"])
    K = args.trajectory

    def energies(ctx):
        _, _, _, e_at, _ = ctx.forces()
        cur = ctx.get_state()
        m = cur["m"]
        ke = 0.5 * float(np.sum(m * (cur["vx"] ** 2 + cur["vy"] ** 2 + cur["vz"] ** 2)))
        pg = -float(np.sum(m * (G[0] * cur["x"] + G[1] * cur["y"] + G[2] * cur["z"])))
        return {"at": e_at, "kinetic": ke, "gravity": pg, "total": e_at + ke + pg}, cur

    out = {}
    for prec in ("mixed", "fp64"):
        ctx = Context(w["algorithm"], prec, w["cutoff"], DT, G, 1.0, device=local, use_graph=True,
                      stream=C.c_void_p(stream.cuda_stream))
        ctx.set_state(st)
        # an untimed run of the same K steps sizes the lists and the chunk-pair queue for the whole
        # trajectory (an overflow inside a K-step call re-runs all K steps) and builds the graph
        ctx.step(K)
        ctx.set_state(st)
        e0, _ = energies(ctx)
        # step 0 alone (the densest step of a run that spreads out)
        step0 = []
        for _ in range(3):
            ctx.set_state(st)
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            c0 = ctx.step(1)
            b.record(stream)
            b.synchronize()
            step0.append(a.elapsed_time(b))
        ctx.set_state(st)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        counts = ctx.step(K)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        eK, final = energies(ctx)
        out[prec] = dict(ms=ms, counts=[int(c) for c in counts], e0=e0, eK=eK, final=final, step0_ms=min(step0),
                         step0_count=int(c0[0]))
        ctx.close()
    mx, fp = out["mixed"], out["fp64"]

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    pos_err = rel(np.stack([mx["final"][k] for k in ("x", "y", "z")]), np.stack([fp["final"][k] for k in ("x", "y", "z")]))
    line = {
        "metric": "triplets/s", "mode": "trajectory", "workload": f"{args.workload}: {w['desc']}", "n": n,
        "steps": K, "data": "synthetic (the reference generator's sequences)",
        "warmup": "one untimed run of the same K steps from the same input, then the timed one",
        "mixed": {"ms_per_step": mx["ms"] / K, "value": sum(mx["counts"]) / (mx["ms"] * 1e-3),
                  "triplets_first_last": [mx["counts"][0], mx["counts"][-1]],
                  "step0_ms": mx["step0_ms"], "step0_triplets_per_s": mx["step0_count"] / (mx["step0_ms"] * 1e-3)},
        "fp64": {"ms_per_step": fp["ms"] / K, "value": sum(fp["counts"]) / (fp["ms"] * 1e-3),
                 "triplets_first_last": [fp["counts"][0], fp["counts"][-1]],
                 "step0_ms": fp["step0_ms"], "step0_triplets_per_s": fp["step0_count"] / (fp["step0_ms"] * 1e-3)},
        "speedup_mixed_vs_fp64": fp["ms"] / mx["ms"],
        "counts_equal_step0": mx["counts"][0] == fp["counts"][0],
        "counts_max_rel_diff": max(abs(a - b) / max(b, 1) for a, b in zip(mx["counts"], fp["counts"])),
        "energy_fp64": {"step0": fp["e0"], f"step{K}": fp["eK"]},
        "energy_mixed": {"step0": mx["e0"], f"step{K}": mx["eK"]},
        "energy_drift_rel": {
            "fp64_total": (fp["eK"]["total"] - fp["e0"]["total"]) / abs(fp["e0"]["total"]),
            "mixed_total": (mx["eK"]["total"] - mx["e0"]["total"]) / abs(mx["e0"]["total"]),
            "mixed_vs_fp64_at_step0": (mx["e0"]["at"] - fp["e0"]["at"]) / abs(fp["e0"]["at"]),
            f"mixed_vs_fp64_at_step{K}": (mx["eK"]["at"] - fp["eK"]["at"]) / abs(fp["eK"]["at"]),
            f"mixed_vs_fp64_total_step{K}": (mx["eK"]["total"] - fp["eK"]["total"]) / abs(fp["eK"]["total"]),
        },
        f"positions_rel_l2_mixed_vs_fp64_step{K}": pos_err,
    }
    print(json.dumps(line), flush=True)


def run_batch(args, local):
    """C5: 64 independent systems, N uniform in 512..4096, each uniform at density 2.048, evaluated
    in one batched call (one set of launches over all systems): mixed-precision forces/energy for
    AUTA (no cutoff) and P3BCA (cutoff 2), and the batched adjoint of a force-matching loss
    sum |f_mixed(nu) - f_FP64(1.1 nu)|^2 (gradients w.r.t. positions and nu).  Times are CUDA
    events around the C-ABI calls, host-array copies included."""
    import torch
    from threebodymdalgorithms_b200 import Context, generators

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    systems = generators.batch_of_systems(64, 512, 4096, 2.048)
    offsets, cat = generators.pack_systems(systems)

    def timed(fn, reps):
        out = None
        ms = []
        for _ in range(reps):
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return out, min(ms)

    res = {}
    for algo, cut in (("p3bca", 2.0), ("auta", 0.0)):
        mx = Context(algo, "mixed", cut, stream=C.c_void_p(stream.cuda_stream))
        ref = Context(algo, "fp64", cut, nu=1.1, stream=C.c_void_p(stream.cuda_stream))
        reps = max(1, min(args.steps, 3 if algo == "auta" else 20))
        fwd = lambda: mx.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
        fwd()
        (fx, fy, fz, e, cnt), f_ms = timed(fwd, reps)
        target = ref.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
        g = [2.0 * (a - b) for a, b in zip((fx, fy, fz), target[:3])]
        ge = np.zeros(len(systems))
        adj = lambda: mx.batch_adjoint(offsets, cat["x"], cat["y"], cat["z"], g[0], g[1], g[2], ge)
        adj()
        _, a_ms = timed(adj, reps)
        trips = int(cnt.sum())
        res[algo] = {"cutoff": cut, "triplets": trips, "forward_ms": f_ms, "forward_triplets_per_s": trips / (f_ms * 1e-3),
                     "adjoint_ms": a_ms, "adjoint_triplets_per_s": trips / (a_ms * 1e-3), "repeats": reps}
        mx.close()
        ref.close()
    line = {"metric": "triplets/s", "mode": "batched", "workload": "c5: 64 systems, N uniform in 512..4096, density 2.048",
            "n_systems": 64, "n_total": int(offsets[-1]), "precision": "mixed (FP64 target forces at 1.1 nu)",
            "data": "synthetic (seeded uniform systems)", "timing": "CUDA events around the batched C-ABI calls, "
            "host copies included; best of the repeats", **res}
    print(json.dumps(line), flush=True)


def cpu_baseline(w, st):
    """The oracle (OpenMP restatement of the reference loop with a cell list) on this host's cores,
    one full step of the workload (bounded: about 1-20 s)."""
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    if w["algorithm"] == "p3bca":
        sample = dict(st)
        label = f"one full step of the workload (N={len(st['x'])})"
    else:
        k = min(len(st["x"]), 1024)
        sample = {key: v[:k] for key, v in st.items()}
        label = f"first {k} particles of the workload, one step"
    t = time.perf_counter()
    _, counts = O.simulate(w["algorithm"], 1, sample, DT, G, w["cutoff"], 1.0, nthreads=cores)
    dt = time.perf_counter() - t
    return {"value": float(counts[0]) / dt, "unit": "triplets/s", "cores": cores, "kind": "port", "sample": label,
            "seconds": dt}


def run_reference(args, world, rank):
    """The reference's own CPU code (built from its sources into oracle/_ref) on a bounded sample
    of the workload: a cube of the workload's particles at the same density and cutoff, sized so
    one step takes a few seconds.  Its loop is O(N^3) in candidates, so the full-size step is
    extrapolated by the candidate count C(N,3)/C(n,3) and both numbers are reported."""
    if rank != 0:
        return
    from oracle import oracle as O
    w = WORKLOADS[args.workload]
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference built from its sources) "
                          "is missing on this machine"}), flush=True)
        return
    st = make_input(w)
    N = len(st["x"])
    budget = min(10.0, 150.0 / max(args.steps + args.warmup, 1))

    def sample(k):
        if w["algorithm"] == "p3bca":
            d = (st["x"] - st["x"].min()) ** 2 + (st["y"] - st["y"].min()) ** 2 + (st["z"] - st["z"].min()) ** 2
            idx = np.sort(np.argsort(d, kind="stable")[:k])  # a corner chunk at the workload's density
        else:
            idx = np.arange(min(k, N))
        return {key: v[idx] for key, v in st.items()}

    from concurrent.futures import ThreadPoolExecutor
    from threebodymdalgorithms_b200 import csvio
    cores = os.cpu_count() or 1

    def run(s, copies=1):
        """One reference step on sample s in `copies` concurrent processes (the reference is one MPI
        rank per process; there is no MPI here, so every core runs its own rank of the same step).
        Returns (triplets of one copy, slowest copy's own step time)."""
        with tempfile.TemporaryDirectory() as tmp:
            path = str(Path(tmp) / "in.csv")
            csvio.write_input(path, s)
            with ThreadPoolExecutor(copies) as ex:
                res = list(ex.map(lambda _: O.reference_dump(path, w["algorithm"], "sim", 1, DT, G, w["cutoff"], 1.0),
                                  range(copies)))
        return int(res[0][1][0]), max(r[2] for r in res)

    k = 256
    _, secs = run(sample(k))
    rate = math.comb(k, 3) / max(secs, 1e-6)  # candidate triplets per second
    while k < N and math.comb(2 * k, 3) / rate < budget:
        k *= 2
    k = min(k, N)
    s = sample(k)
    for _ in range(args.warmup):
        run(s, cores)
    trips, total = 0, 0.0
    for _ in range(args.steps):
        c, secs = run(s, cores)
        trips += c * cores  # every core evaluated the sample's triplets
        total += secs
    sample_rate = trips / total
    per_step_sample = total / args.steps / cores  # one step of the sample with all cores sharing it
    full_trip = WORKLOAD_TRIPLETS.get(args.workload)
    ext_step = per_step_sample * math.comb(N, 3) / math.comb(k, 3)
    value = (full_trip / ext_step) if full_trip else sample_rate
    line = {"impl": "reference", "metric": "triplets/s", "value": value, "unit": "triplets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ext_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {w['desc']}", "algorithm": w["algorithm"], "n": N,
                       "cutoff": w["cutoff"]},
            "cpu_baseline": {"value": value, "unit": "triplets/s", "cores": cores, "kind": "reference",
                             "sample": f"{k} particles of the workload (same density/cutoff), the reference's O(N^3) "
                                       f"loop in {cores} concurrent single-rank processes (no MPI on this host; the "
                                       f"aggregate is the ideal {cores}-rank rate): {sample_rate:.4g} triplets/s on "
                                       f"the sample; the full step extrapolated by C(N,3)/C(n,3)"},
            "sample_value": sample_rate,
            "e2e": {"value": value, "unit": "triplets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# exact triplets per step of the full workloads (from the oracle; C1/C2 are C(N,3))
WORKLOAD_TRIPLETS = {"c1": math.comb(512, 3), "c2": math.comb(8192, 3), "c3": 48272380, "c3c15": 8583257,
                     "c4": 7282646752}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="c3")
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 run beside the mixed one")
    ap.add_argument("--trajectory", type=int, default=0,
                    help="instead of the headline line: a K-step run (one graph-replayed call), mixed vs FP64, "
                         "with energies at step 0 and K")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    if args.trajectory > 0:
        run_trajectory(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.workload == "c5":
        run_batch(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
