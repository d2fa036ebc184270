#!/usr/bin/env python3
"""Benchmark of the B200-native Zebraflow hot path.

Default workload: the periodic Y-bifurcation of 256x256x1024 lattice points
(parent radius 30 splitting at 40 degrees into daughters of radius 22, about
3.1M fluid points), halfway bounce-back walls, uniform Guo force 2e-6 along
the parent axis, fp32 populations.  A step is one LBM time step
(pull stream + BGK/Guo collision + walls) over the whole vessel.

One JSON line on rank 0:
  value  MLUPS with populations resident in HBM, device-timed with CUDA
         events on the stream the kernels run on (max over ranks)
  e2e    the same metric through the C ABI with host buffers: every step
         sets the uniform force from pinned host memory and reads the FP64
         global mass back to the host
  roofline, cpu_baseline, clocks, gpu_launches as described in DESIGN.md.

``--impl reference`` times the CPU restatement of the reference algorithm
(two LBM passes, FEQ store, F_OLD copy; OpenMP) on the host cores instead.
Input data are synthetic (seeded geometry); there is no dataset.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (nx, ny, nz, Rp, Rd, half_angle, g)
    "bifurcation_256x256x1024": (256, 256, 1024, 30.0, 22.0, 20.0, 2e-6),
    "bifurcation_x2_256x256x1024": (256, 256, 1024, 60.0, 44.0, 20.0, 2e-6),
    "bifurcation_small_128x96x256": (128, 96, 256, 15.0, 11.0, 20.0, 2e-6),
}
BYTES_PER_LUP = {0: 152, 1: 76, 2: 76, 3: 152}  # 2*19*S, S = bytes per stored population
DTYPE_NAME = {0: "f32", 1: "f16-storage/f32-math", 2: "bf16-storage/f32-math",
              3: "f32-deviation-storage/f32-math"}


def read_peaks():
    for path in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        try:
            with open(path) as fh:
                pk = json.load(fh)
            return float(pk["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def read_traffic(workload, storage):
    """DRAM bytes per fluid-point update of k_lbm from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_lbm_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d[DTYPE_NAME[storage]]["dram_bytes_per_fluid_point"])
    except Exception:
        return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_geometry(name):
    import zebraflow_b200 as zf
    nx, ny, nz, Rp, Rd, ang, g = WORKLOADS[name]
    b, layout = zf.gen_bifurcation(nx, ny, nz, Rp, Rd, ang)
    return b, (nx, ny, nz, Rp, Rd, ang, g), layout


def cpu_reference_time(b, dims, storage, max_seconds=15.0, threads=None):
    """Times the reference-faithful CPU restatement (oracle port, fp32) on the
    host cores: returns (MLUPS, cores, sample description)."""
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle.bind import OracleLBM
    nx, ny, nz, Rp, Rd, ang, g = dims
    o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.9, g=(0, 0, g), precision="f32",
                  faithful=True)
    n_fluid = int((b > 0).sum())
    o.time_steps(2)  # warm-up (first touch of the arrays)
    steps, spent = 0, 0.0
    per = max(1, int(o.time_steps(1) > 0))
    t_budget = max_seconds
    while spent < t_budget:
        dt = o.time_steps(per)
        steps += per
        spent += dt
        if dt < 0.5:
            per *= 2
    o.close()
    mlups = n_fluid * steps / spent / 1e6
    return mlups, steps, spent


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    b, dims, _ = build_geometry(args.workload)
    n_fluid = int((b > 0).sum())
    from oracle.bind import OracleLBM
    nx, ny, nz, Rp, Rd, ang, g = dims
    o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.9, g=(0, 0, g), precision="f32",
                  faithful=True)
    for _ in range(min(args.warmup, 5)):
        o.time_steps(1)
    # each step is the full workload; the number of timed steps is bounded so
    # the run stays within about two minutes of host time
    t1 = o.time_steps(1)
    nsteps = max(1, min(args.steps, int(120.0 / max(t1, 1e-6))))
    times = [o.time_steps(1) for _ in range(nsteps)]
    o.close()
    t = sum(times)
    mlups = n_fluid * nsteps / t / 1e6
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * t / nsteps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "fluid_points": n_fluid, "wall": "halfway bounce-back",
                   "storage": "f32", "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": int(os.environ["OMP_NUM_THREADS"]),
                         "kind": "port",
                         "sample": f"{nsteps} full LBM steps of the workload (of {args.steps} asked; "
                                   f"bounded to ~2 min of host time)"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    import torch.distributed as dist
    import zebraflow_b200 as zf

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    b, dims, layout = build_geometry(args.workload)
    nx, ny, nz, Rp, Rd, ang, g = dims
    storage = {"f32": zf.STORE_F32, "f16": zf.STORE_F16, "bf16": zf.STORE_BF16,
               "f32dev": zf.STORE_F32_DEV}[args.storage]
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.9, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), storage=storage,
                          g=(0.0, 0.0, g))
    ctx = zf.Context(p, device=dev)
    ctx.set_lattice(b)
    n_fluid = ctx.n_fluid
    stream = torch.cuda.current_stream(dev)
    zf.lib().zf_set_stream(ctx._h, C_void(stream.cuda_stream))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # warm-up (also develops the flow a little)
    for _ in range(args.warmup):
        ctx.lbm_step(store_moments=False)
    barrier()

    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        ctx.lbm_step(store_moments=False)
    ev1.record(stream)
    barrier()
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop() if sampler else None

    # end-to-end through the C ABI with host buffers
    gh = torch.tensor([0.0, 0.0, g], dtype=torch.float32).pin_memory()
    import ctypes
    mass = ctypes.c_double()
    e2e_steps = max(1, min(args.steps, 50))
    barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        zf.lib().zf_set_uniform_force(ctx._h, ctypes.cast(gh.data_ptr(), ctypes.POINTER(ctypes.c_float)))
        rc = zf.lib().zf_lbm_step_mass(ctx._h, 0, 0, ctypes.byref(mass))
        if rc:
            raise zf.ZfError(rc, zf.lib().zf_last_error().decode())
    e1.record(stream)
    barrier()
    wall_e2e = time.perf_counter() - t0
    ms_e2e = max(e0.elapsed_time(e1), 1e3 * wall_e2e)
    zf.lib().zf_set_stream(ctx._h, None)

    # max over ranks
    if world > 1:
        t = torch.tensor([ms, ms_e2e], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])

    mlups = world * n_fluid * args.steps / (ms * 1e-3) / 1e6
    mlups_e2e = world * n_fluid * e2e_steps / (ms_e2e * 1e-3) / 1e6
    peak, peak_kind = read_peaks()
    bytes_lup = BYTES_PER_LUP[storage]
    achieved = n_fluid * bytes_lup / (ms * 1e-3 / args.steps) / 1e9
    traffic = read_traffic(args.workload, storage)

    result = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            mlups_cpu, csteps, cspent = cpu_reference_time(b, dims, storage, max_seconds=args.cpu_seconds,
                                                           threads=threads)
            cpu = {"value": round(mlups_cpu, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                   "sample": f"{csteps} full LBM steps of the same workload (fp32, reference pass "
                             f"structure) in {cspent:.1f} s"}
        result = {
            "metric": "MLUPS", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_NAME[storage],
            "data": "synthetic",
            "config": {"workload": args.workload, "fluid_points": int(n_fluid),
                       "wall": "halfway bounce-back", "tau": 0.9, "g": g,
                       "storage": args.storage, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (populations %.0f MB per step)" % (n_fluid * bytes_lup / 1e6)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": None if traffic is None else round(traffic * n_fluid),
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": n_fluid * bytes_lup},
            "cpu_baseline": cpu,
            "e2e": {"value": round(mlups_e2e, 1), "unit": "MLUPS", "h2d_bytes_per_step": 12,
                    "d2h_bytes_per_step": 8},
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
        print(json.dumps(result), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def C_void(ptr):
    import ctypes
    return ctypes.c_void_p(ptr)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bifurcation_256x256x1024", choices=sorted(WORKLOADS))
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f32dev"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
