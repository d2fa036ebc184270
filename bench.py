#!/usr/bin/env python3
"""Benchmark of the B200-native Zebraflow time step (LBM + IB + membranes).

Default workload ``c1_bifurcation_256x256x1024_2000rbc``: the periodic
Y-bifurcation of 256x256x1024 lattice points (parent radius 30 splitting at
40 degrees into daughters of radius 22, about 3.1M fluid points), halfway
bounce-back walls, tau 0.9, uniform Guo force 2e-6 along the parent axis,
2000 nucleated RBCs (icosphere membranes of 642 nodes / 1280 triangles scaled
to semi-axes 7, 4.5, 2 lattice units, nuclei of 162 nodes scaled to 2.5, 1.8,
1.2) placed from a seed, a marching-tetrahedra wall mesh of the vessel.

A bench step is one cycle of the reference time loop (ZebraflowWT.c:5646-12190
with SOLVERSTAGGER = 50, :151): 50 LBM iterations, the 50th of which also runs
the membrane forces, IB velocity interpolation with wall repulsion,
nucleus-membrane and cell-cell repulsion, IB spreading and the position
update.  Every warm-up and every timed step therefore contains exactly one
membrane/IB block, so that ``--steps K`` times K whole cycles.

One JSON line on rank 0:
  value   MLUPS of the coupled step (fluid points x LBM iterations / time),
          state resident in HBM, device-timed with CUDA events on the stream
          the kernels run on (max over ranks); ``membrane_node_updates_per_s``
          (membrane + nucleus nodes x membrane blocks / time) beside it
  e2e     the same metric through the C ABI with host buffers: every step
          sets the driving force from pinned host memory, and reads the FP64
          global mass and every cell's node positions and status back into
          pinned host memory (what a host-side caller of the membrane step,
          such as the reference's cell management, needs each cycle)
  roofline  k_lbm's algorithmic bytes (2 x 19 populations x bytes each per
          fluid point) over its average launch time, from CUDA events around
          the runs of plain LBM launches in a second, profiled pass of the
          same steps; ``membrane`` beside it: the membrane/IB block's stage
          times and its bytes per membrane-node update
  storage_variants  the same measurement with fp16 / bf16 deviation storage
  cpu_baseline  the CPU restatement of the reference time loop (oracle,
          OpenMP, reference pass structure) on the host cores, one bounded
          sample of whole cycles

``--impl reference`` times that CPU restatement alone, as the reference arm,
and beside it (``reference_code_lbm``) the reference's own LBM blocks, compiled
from its source by oracle/ref/Makefile, on the part of the lattice that fits
the reference's compile-time box.  It builds its inputs with the generators
compiled into oracle/liboracle.so and does not load the GPU library.
Input data are synthetic (seeded geometry and cells); there is no dataset.
"""
from __future__ import annotations

import argparse
import ctypes
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
    # name: (nx, ny, nz, Rp, Rd, half_angle_deg, g, cells)
    "c1_bifurcation_256x256x1024_2000rbc": (256, 256, 1024, 30.0, 22.0, 20.0, 2e-6, 2000),
    # the same box with radii doubled: the ~12 M fluid nodes the workload's
    # description states (12,047,196), and 8000 cells for about its 20 % hematocrit
    "c1x2_bifurcation_256x256x1024_r60_8000rbc": (256, 256, 1024, 60.0, 44.0, 20.0, 2e-6, 8000),
    "bifurcation_small_128x96x256_60rbc": (128, 96, 256, 15.0, 11.0, 20.0, 2e-6, 60),
}
DX_UM = 0.5
STAGGER = 50                      # SOLVERSTAGGER, ZebraflowWT.c:151
WALL_HALFWAY_BB = 0
AXES_UM = (3.5, 2.25, 1.0)        # 7, 4.5, 2 lattice units
AXES_N_UM = (1.25, 0.9, 0.6)      # 2.5, 1.8, 1.2 lattice units
# placement margin (um) around each cell's ellipsoid: adjacent cells start
# about 1 um apart, outside the reference's repulsion range, so that no cell
# starts inside another's repulsion zone
PLACEMENT_MARGIN_UM = 0.4
STORAGES = {"f32": 0, "f16": 1, "bf16": 2, "f32dev": 3}
BYTES_PER_POP = {0: 4, 1: 2, 2: 2, 3: 4}
DTYPE_NAME = {0: "f32", 1: "f16-storage/f32-math", 2: "bf16-storage/f32-math",
              3: "f32-deviation-storage/f32-math"}


def lbm_bytes_per_point(storage: int) -> int:
    """Algorithmic DRAM bytes of one fluid-point update of the LBM step: the
    19 populations read and the 19 written (152 B fp32, 76 B fp16/bf16)."""
    return 2 * 19 * BYTES_PER_POP[storage]


# bytes k_lbm moves per fluid point beyond the populations: the link word
# (4 B) and the body force (12 B); on membrane iterations also the 4 moments
# written and the force cleared (28 B)
LBM_OVERHEAD_BYTES = {"plain_iteration": 16, "membrane_iteration": 44}


def membrane_bytes_per_node(n_node: int, footprint: float = 1000.0) -> float:
    """Algorithmic bytes of one membrane-node update of the membrane/IB block:
    B_mn = 72 + 36 L/N, with 72 B of position, velocity and force traffic per
    node and 36 B (12 B velocity read, 24 B force read-modify-write) per
    lattice point of a cell's IB footprint, L of them (about 1000 for the
    7 x 4.5 x 2 lattice-unit ellipsoid) shared by its N nodes."""
    return 72.0 + 36.0 * footprint / n_node


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(workload, storage):
    """DRAM bytes per fluid-point update of k_lbm from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_lbm_traffic.json")) as fh:
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
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_median": statistics.median(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(vals, device):
    """Element-wise maximum of a list of floats over all ranks (timings are
    reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Case:
    """Seeded geometry of one workload: lattice, wall mesh, cell meshes, cells.
    `inputs` is the generator binding (zebraflow_b200.inputs() by default; the
    reference arm passes oracle.bind.inputs(), the same generators compiled
    into the CPU library)."""

    def __init__(self, name, n_cells=None, seed=2024, inputs=None):
        from zebraflow_b200 import mesh_edges
        if inputs is None:
            import zebraflow_b200 as zf
            inputs = zf.inputs()
        self.gen = inputs
        nx, ny, nz, Rp, Rd, ang, g, nc = WORKLOADS[name]
        if n_cells is None:
            n_cells = nc
        self.name, self.dims, self.g, self.seed = name, (nx, ny, nz), g, seed
        self.b, self.layout = inputs.gen_bifurcation(nx, ny, nz, Rp, Rd, ang)
        self.n_fluid = int((self.b > 0).sum())
        self.mesh = self.cells = self.wall = None
        self.n_cells = 0
        if n_cells > 0:
            self.wall = inputs.gen_wall_bifurcation(nx, ny, nz, Rp, Rd, ang, dx=DX_UM)
            xyz, tri = inputs.gen_icosphere(3)
            xyzn, trin = inputs.gen_icosphere(2)
            rest = xyz * np.array(AXES_UM)
            rest_n = xyzn * np.array(AXES_N_UM)
            self.mesh = (rest, tri, rest_n, mesh_edges(trin))
            self.cells = inputs.gen_cells(self.b, n_cells, rest, rest_n, AXES_UM, seed=seed, dx=DX_UM,
                                          margin=PLACEMENT_MARGIN_UM)
            self.n_requested = n_cells
            self.n_cells = self.cells[0].shape[1]
            self.nn, self.nnn = rest.shape[0], rest_n.shape[0]
            vol_cell = 4.0 / 3.0 * np.pi * np.prod(np.array(AXES_UM) / DX_UM)
            self.hematocrit = self.n_cells * vol_cell / self.n_fluid

    def params(self, storage: int):
        nx, ny, nz = self.dims
        return self.gen.default_params(nx=nx, ny=ny, nz=nz, tau=0.9, tau_from_phase=0,
                                       wall_mode=WALL_HALFWAY_BB, periodic=(0, 0, 1), storage=storage,
                                       g=(0.0, 0.0, self.g), origin=(0.0, 0.0, 0.0), dx=DX_UM,
                                       area0=0.0, volume0=0.0)

    @property
    def n_nodes(self):
        return self.n_cells * (self.nn + self.nnn) if self.n_cells else 0

    def config(self, storage_name):
        c = {"workload": self.name, "lattice": "x".join(map(str, self.dims)),
             "fluid_points": self.n_fluid, "wall": "halfway bounce-back", "tau": 0.9,
             "g": self.g, "storage": storage_name, "l2": "inputs larger than L2",
             "step": f"one cycle of the reference loop: {STAGGER} LBM iterations, the last with "
                     f"the membrane/IB block"}
        if self.n_cells:
            c.update({"cells": self.n_cells, "cells_requested": self.n_requested,
                      "placement_margin_um": PLACEMENT_MARGIN_UM,
                      "membrane_nodes": self.nn, "nucleus_nodes": self.nnn,
                      "hematocrit": round(float(self.hematocrit), 3), "stagger": STAGGER,
                      "wall_mesh_triangles": int(self.wall[1].shape[1]), "seed": self.seed,
                      "moduli": "reference SI constants"})
        return c

    def oracle_world(self, precision="f32"):
        """The CPU restatement of the reference loop on the same inputs."""
        from oracle.bind import OracleCells, OracleLBM, OracleWorld
        p = self.params(0)
        lbm = OracleLBM(self.b, wall_mode=0, periodic=(0, 0, 1), tau=0.9, g=(0.0, 0.0, self.g),
                        precision=precision, faithful=True)
        if not self.n_cells:
            return lbm, None, None
        oc = OracleCells(*self.mesh, p, precision=precision)
        oc.set_cells(*self.cells)
        w = OracleWorld(lbm, oc, p)
        w.set_wall(*self.wall)
        return lbm, oc, w


def oracle_threads():
    from oracle.bind import lib as olib
    try:
        return int(olib().orc_max_threads())
    except Exception:
        return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def time_oracle(case, max_seconds, max_cycles, stagger=STAGGER):
    """Times the CPU restatement: 3 LBM warm-up iterations, then whole blocks
    of the time loop (each ending in a membrane iteration; the first block
    completes the warm-up cycle) until max_seconds or max_cycles blocks.
    Returns (LBM iterations, membrane blocks, seconds)."""
    lbm, oc, w = case.oracle_world()
    run = (lambda n: w.step(n)) if w is not None else (lambda n: lbm.time_steps(n))
    run(3)
    it, steps, blocks, spent = 3, 0, 0, 0.0
    while True:
        n = stagger - it % stagger
        if blocks > 0 and (spent >= max_seconds or blocks >= max_cycles):
            break
        t0 = time.perf_counter()
        run(n)
        spent += time.perf_counter() - t0
        it += n
        steps += n
        blocks += 1
    for o in (w, oc, lbm):
        if o is not None:
            o.close()
    return steps, (blocks if w is not None else 0), spent


# the reference's compile-time lattice box (ZebraflowWT.c:81-83): IM, JM, KM
REF_BOX = (249, 547, 723)


def time_reference_code(case, max_seconds, max_steps):
    """Times the reference's own LBM step (its stream-collide, wall and copy
    blocks of main(), run by oracle/_ref/ref_time; oracle/ref/Makefile builds
    it from ZebraflowWT.c) on the part of the workload's lattice that fits the
    reference's compile-time box, the cut planes closed by walls.  Returns a
    dict for the JSON line, or None when the program was not built."""
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_time")
    if not os.path.exists(exe):
        return None
    nx, ny, nz = case.b.shape
    s = np.array(case.b[:min(nx, REF_BOX[0] - 1), :min(ny, REF_BOX[1] - 1), :min(nz, REF_BOX[2] - 3)],
                 np.int32)
    for sl in ((slice(None), slice(None), 0), (slice(None), slice(None), -1),
               (0, slice(None), slice(None)), (-1, slice(None), slice(None)),
               (slice(None), 0, slice(None)), (slice(None), -1, slice(None))):
        pl = s[sl]
        pl[pl > 0] = 0
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "lattice.bin")
        with open(path, "wb") as fh:
            fh.write(np.array(s.shape, np.int32).tobytes())
            fh.write(s.tobytes())
        out = subprocess.run([exe, path, str(max_steps), str(max_seconds)], capture_output=True,
                             text=True, timeout=max_seconds + 600)
    if out.returncode != 0:
        return {"unavailable": f"ref_time exited {out.returncode}: {out.stderr.strip()[-200:]}"}
    fluid, steps, t, threads = out.stdout.strip().split("\n")[-1].split()
    fluid, steps, t, threads = int(fluid), int(steps), float(t), int(threads)
    return {"value": round(fluid * steps / t / 1e6, 3), "unit": "MLUPS", "cores": threads,
            "kind": "reference",
            "sample": f"{steps} LBM steps of the reference's own code on the first "
                      f"{'x'.join(map(str, s.shape))} points of the lattice ({fluid} fluid points; "
                      f"the reference box holds no more), after 3 warm-up steps; LBM step only"}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from oracle.bind import inputs as oracle_inputs
    case = Case(args.workload, args.cells, args.seed, inputs=oracle_inputs())
    steps, mem, t = time_oracle(case, args.reference_seconds, args.steps)
    mlups = case.n_fluid * steps / t / 1e6
    cores = oracle_threads()
    cycles = steps / STAGGER
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * t / cycles, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "parallelism": f"host OpenMP x{cores}",
        "membrane_node_updates_per_s": round(case.n_nodes * mem / t, 1),
        "config": case.config("f32"),
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
                         "sample": f"{steps} LBM iterations ({mem} with the membrane/IB block) of the "
                                   f"workload after 3 warm-up iterations, {args.steps} cycles asked; "
                                   f"bounded to ~{args.reference_seconds:.0f} s of host time"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    ref = time_reference_code(case, min(30.0, args.reference_seconds), max(args.steps, 10))
    if ref is not None:
        # the compiled reference's own LBM blocks beside the restatement's coupled step
        line["reference_code_lbm"] = ref
    print(json.dumps(line), flush=True)
    return 0


def measure_storage(case, storage, args, dev, stream, barrier, sample_clocks=False):
    """Warm-up, timed pass, profiled pass (per-launch and per-stage events)
    and the e2e pass for one storage form.  Every pass runs whole cycles of
    STAGGER iterations from an iteration count that is a multiple of
    STAGGER, so each cycle ends in one membrane/IB block.  Returns a dict of
    raw figures."""
    import torch
    import zebraflow_b200 as zf

    ctx = zf.Context(case.params(storage), device=dev)
    ctx.set_lattice(case.b)
    if case.n_cells:
        ctx.set_wall(*case.wall)
        ctx.set_mesh(*case.mesh)
        ctx.set_cells(*case.cells)
    ctx.set_stream(stream.cuda_stream)
    S = ctx.params.stagger
    assert S == STAGGER
    K = args.steps

    ctx.step(S * args.warmup)
    barrier()
    sampler = ClockSampler(dev) if sample_clocks else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    assert ctx.iteration() % S == 0
    l0 = ctx.launch_count()
    barrier()
    ev0.record(stream)
    ctx.step(S * K)
    ev1.record(stream)
    barrier()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launch_count() - l0
    clocks = sampler.stop() if sampler else None
    n_mem = K if case.n_cells else 0

    # second pass with per-launch and per-stage events
    ctx.profile(True, S * K + 8)
    barrier()
    ev0.record(stream)
    ctx.step(S * K)
    ev1.record(stream)
    barrier()
    ms_prof = ev0.elapsed_time(ev1)
    lbm_ms, lbm_n, mem_ms, mem_n = ctx.profile_read()
    stages, blocks = ctx.profile_stages()
    ctx.profile(False)

    # end to end through the C ABI with host buffers in pinned memory: each
    # cycle sets the force from the host, runs, and reads back the mass, the
    # node positions and the cell status.  The positions and statuses are
    # copied with zf_get_cells_async, so the copy of one cycle's state runs
    # beside the next cycle's LBM iterations (the next membrane iteration
    # waits for it); the last copy is waited for inside the timed region.
    L = zf.lib()
    gh = torch.tensor([0.0, 0.0, case.g], dtype=torch.float32).pin_memory()
    gptr = ctypes.cast(gh.data_ptr(), ctypes.POINTER(ctypes.c_float))
    mass = ctypes.c_double()
    d2h = 8
    if case.n_cells:
        hx = torch.empty(3 * case.n_cells * case.nn, dtype=torch.float64).pin_memory()
        hxn = torch.empty(3 * case.n_cells * case.nnn, dtype=torch.float64).pin_memory()
        hst = torch.empty(case.n_cells, dtype=torch.int32).pin_memory()
        d2h += (hx.numel() + hxn.numel()) * 8 + hst.numel() * 4
        px, pxn, pst = (ctypes.c_void_p(t.data_ptr()) for t in (hx, hxn, hst))

    def e2e_cycle():
        rc = L.zf_set_uniform_force(ctx._h, gptr)
        if not rc and S > 1:
            rc = L.zf_step(ctx._h, S - 1)
        if not rc:
            rc = L.zf_step_mass(ctx._h, ctypes.byref(mass))
        if not rc and case.n_cells:
            rc = L.zf_get_cells_async(ctx._h, px, pxn, pst)
        if rc:
            raise zf.ZfError(rc, L.zf_last_error().decode())

    def e2e_wait():
        if case.n_cells:
            rc = L.zf_wait_cells(ctx._h)
            if rc:
                raise zf.ZfError(rc, L.zf_last_error().decode())

    e2e_cycle()  # first use of the pinned buffers, untimed
    e2e_wait()
    barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        e2e_cycle()
    e2e_wait()
    barrier()
    ms_e2e = 1e3 * (time.perf_counter() - t0)
    removed_end = int(ctx.status().cells_removed)
    # wall shear stress of the final state (compared across storage forms)
    wss = ctx.wss()[0] if case.wall is not None else None
    ctx.set_stream(None)
    ctx.close()
    return {"ms": ms, "launches": launches, "clocks": clocks, "n_mem": n_mem, "removed_end": removed_end,
            "ms_prof": ms_prof, "lbm_ms": lbm_ms, "lbm_n": lbm_n, "mem_ms": mem_ms, "mem_n": mem_n,
            "stages": stages, "blocks": blocks, "ms_e2e": ms_e2e, "d2h": d2h, "wss": wss,
            "mass": mass.value}


def summarize(case, storage, r, steps, world, peak):
    """Figures of one storage form from the raw times of measure_storage."""
    n = case.n_fluid
    its = steps * STAGGER
    out = {"mlups": world * n * its / (r["ms"] * 1e-3) / 1e6,
           "ms_per_step": r["ms"] / steps,
           "mlups_e2e": world * n * its / (r["ms_e2e"] * 1e-3) / 1e6}
    out["membrane_node_updates_per_s"] = world * case.n_nodes * r["n_mem"] / (r["ms"] * 1e-3)
    # k_lbm roofline from the profiled pass: algorithmic bytes of the plain LBM
    # launches (timed as runs of consecutive launches) over their device time
    alg = n * lbm_bytes_per_point(storage) * r["lbm_n"]
    lbm_s = r["lbm_ms"] * 1e-3
    out["k_lbm_ms"] = r["lbm_ms"] / max(r["lbm_n"], 1)
    out["k_lbm_gbs"] = alg / lbm_s / 1e9 if lbm_s > 0 else None
    out["k_lbm_frac"] = out["k_lbm_gbs"] / peak if out["k_lbm_gbs"] else None
    out["membrane_block_ms"] = r["mem_ms"] / r["mem_n"] if r["mem_n"] else None
    out["lbm_share"] = r["lbm_ms"] / r["ms_prof"] if r["ms_prof"] else None
    out["membrane_share"] = r["mem_ms"] / r["ms_prof"] if r["ms_prof"] and r["mem_n"] else None
    return out


class StreamTimer:
    """Times one call of the context's API with CUDA events recorded on the
    stream its kernels run on, synchronised on both sides."""

    def __init__(self, stream, barrier):
        import torch
        self.stream, self.barrier = stream, barrier
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)
        self.seconds = None

    def __call__(self, fn):
        self.barrier()
        self.e0.record(self.stream)
        out = fn()
        self.e1.record(self.stream)
        self.barrier()
        self.seconds = 1e-3 * self.e0.elapsed_time(self.e1)
        return out


def measure_adjoint(dev, stream, barrier, seed=2024, nsteps=500, t0=300, t1=500, K=50):
    """Cost of the hand-written adjoint on the C3 tube (96x96x512, R = 40,
    200 RBCs at slightly deformed positions): J = mean |WSS| over a
    64-lattice-unit wall patch across steps 300..500, gradients for the
    body-force field, tau, Es and kb, checkpoint every 50 steps; first with
    the cells held at their positions, then with the cells moving (the
    coupled step, membrane iterations every 50 steps, plus dJ/dx_0)."""
    import torch
    import zebraflow_b200 as zf
    nx, ny, nz, R = 96, 96, 512, 40.0
    c = (nx - 1) / 2.0
    b = zf.gen_tube(nx, ny, nz, c, c, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array(AXES_UM)
    rest_n = xyzn * np.array(AXES_N_UM)
    x, xn = zf.gen_cells(b, 200, rest, rest_n, AXES_UM, seed=seed, dx=DX_UM, margin=PLACEMENT_MARGIN_UM)
    rng = np.random.default_rng(seed)
    x = x + 0.02 * rng.standard_normal(x.shape)
    wall = zf.gen_wall_tube(c, c, R, nz)
    z = wall[0][2] / DX_UM
    patch = np.nonzero((z >= 224) & (z < 288))[0].astype(np.int32)
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                          periodic=(0, 0, 1), g=(0.0, 0.0, 2e-6), origin=(0.0, 0.0, 0.0), dx=DX_UM,
                          area0=0.0, volume0=0.0, storage=zf.STORE_F32_DEV)
    ctx = zf.Context(p, device=dev)
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.set_mesh(rest, tri, rest_n, zf.mesh_edges(trin))
    ctx.set_cells(x, xn)
    ctx.set_stream(stream.cuda_stream)
    ctx.wss_objective(nsteps, t0, t1, patch)  # warm-up
    t_fwd = t_adj = float("inf")
    timer = StreamTimer(stream, barrier)
    for _ in range(3):  # fastest of three calls each (CUDA events on the context's stream)
        J = timer(lambda: ctx.wss_objective(nsteps, t0, t1, patch))
        t_fwd = min(t_fwd, timer.seconds)
        Ja, gfb, gtau, gEs, gkb = timer(lambda: ctx.wss_adjoint(nsteps, t0, t1, patch, checkpoint=K))
        t_adj = min(t_adj, timer.seconds)
    # the same objective with the cells moving over the window (10 membrane iterations)
    ctx.adjoint_move_cells(True)
    ctx.wss_objective(nsteps, t0, t1, patch)  # warm-up
    m_fwd = m_adj = float("inf")
    for _ in range(3):
        Jm = timer(lambda: ctx.wss_objective(nsteps, t0, t1, patch))
        m_fwd = min(m_fwd, timer.seconds)
        Jma, mfb, mtau, mEs, mkb = timer(lambda: ctx.wss_adjoint(nsteps, t0, t1, patch, checkpoint=K))
        m_adj = min(m_adj, timer.seconds)
    gx, _ = ctx.adjoint_position_gradient()
    moving = {"forward_ms": round(1e3 * m_fwd, 2), "forward_and_adjoint_ms": round(1e3 * m_adj, 2),
              "gradient_cost_over_forward": round((m_adj - m_fwd) / m_fwd, 3), "membrane_iterations": nsteps // 50,
              "J_pa": Jm, "dJ_dtau": mtau, "dJ_dEs": mEs, "dJ_dkb": mkb, "dJ_dfb_max": float(np.abs(mfb).max()),
              "dJ_dx0_max": float(np.abs(gx).max()),
              "repulsions": "differentiated (wall, nucleus-membrane, RBC-RBC)"}
    ctx.set_stream(None)
    ctx.close()
    return {"workload": "c3_tube_96x96x512_200rbc", "fluid_points": int((b > 0).sum()),
            "steps": nsteps, "objective_window": [t0, t1], "patch_wall_nodes": int(patch.size),
            "checkpoint_interval": K, "storage": "f32dev",
            "forward_ms": round(1e3 * t_fwd, 2), "forward_and_adjoint_ms": round(1e3 * t_adj, 2),
            "gradient_cost_over_forward": round((t_adj - t_fwd) / t_fwd, 3),
            "J_pa": J, "dJ_dtau": gtau, "dJ_dEs": gEs, "dJ_dkb": gkb,
            "dJ_dfb_max": float(np.abs(gfb).max()),
            "cells_moving": moving,
            "timing": "CUDA events on the context's stream around each call, fastest of 3"}


def measure_c4(case, dev, stream, barrier, nsteps=2000, t0=1001, K=50, budget_gb=80.0):
    """C4: the flux-split adjoint on the C1 workload (cells held at their
    placed positions), forward in fp16 deviation storage, against the same
    adjoint with fp32 deviation storage.  J = mean over steps t0..nsteps of
    the share of the axial flux through the +x daughter's mid cross-section;
    checkpoint interval K, whose memory (checkpoints + one segment of states)
    must fit the budget.  Reports both costs and the fp16 gradient's error."""
    import zebraflow_b200 as zf
    nx = case.dims[0]
    z2, z3 = case.layout[1], case.layout[2]
    kp = int(round(0.5 * (z2 + z3)))
    n = (0.0, 0.0, 1.0)
    lst = np.argwhere(case.b >= 0) >> 2  # tiles holding listed points
    n_tiles = int(np.unique((lst[:, 2] * 4096 + lst[:, 1]) * 4096 + lst[:, 0]).size)
    res, grads = {}, {}
    for name, st, esz in (("f32dev", zf.STORE_F32_DEV, 4), ("f16", zf.STORE_F16, 2)):
        ctx = zf.Context(case.params(st), device=dev)
        ctx.set_lattice(case.b)
        if case.n_cells:
            ctx.set_wall(*case.wall)
            ctx.set_mesh(*case.mesh)
            ctx.set_cells(*case.cells)
        ctx.set_stream(stream.cuda_stream)
        dom = ctx.domlist()
        fluid = case.b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
        plane = fluid & (dom[:, 2] == kp)
        cx = 0.5 * (nx - 1)
        p0 = np.nonzero(plane & (dom[:, 0] > cx))[0].astype(np.int32)
        p1 = np.nonzero(plane & (dom[:, 0] < cx))[0].astype(np.int32)
        ctx.flux_objective(20, 1, 20, p0, n, p1, n)  # warm-up
        t_fwd = t_adj = float("inf")
        timer = StreamTimer(stream, barrier)
        for _ in range(2):  # faster of two calls each (CUDA events on the context's stream)
            J = timer(lambda: ctx.flux_objective(nsteps, t0, nsteps, p0, n, p1, n))
            t_fwd = min(t_fwd, timer.seconds)
            Ja, g, gtau, gEs, gkb = timer(lambda: ctx.flux_adjoint(nsteps, t0, nsteps, p0, n, p1, n,
                                                                   checkpoint=K))
            t_adj = min(t_adj, timer.seconds)
        ctx.set_stream(None)
        ctx.close()
        grads[name] = g.astype(np.float64)
        # checkpoints and one segment of states, [tile][19][64] populations per state
        states = -(-nsteps // K) + K + 1
        res[name] = {"J": J, "forward_ms": round(1e3 * t_fwd, 2), "forward_and_adjoint_ms": round(1e3 * t_adj, 2),
                     "gradient_cost_over_forward": round((t_adj - t_fwd) / t_fwd, 3), "dJ_dtau": gtau,
                     "dJ_dEs": gEs, "dJ_dkb": gkb,
                     "checkpoint_memory_gb": round(states * 19 * 64 * n_tiles * esz / 1e9, 2)}
    g32, g16 = grads["f32dev"], grads["f16"]
    return {"workload": case.name + "_flux_split", "steps": nsteps, "objective_window": [t0, nsteps],
            "plane_k": kp, "checkpoint_interval": K, "memory_budget_gb": budget_gb,
            "f32dev": res["f32dev"], "f16": res["f16"],
            "f16_rel_l2_error_dJ_dfb": float(np.linalg.norm(g16 - g32) / np.linalg.norm(g32)),
            "f16_rel_error_J": abs(res["f16"]["J"] - res["f32dev"]["J"]) / abs(res["f32dev"]["J"]),
            "timing": "CUDA events on the context's stream around each call, faster of 2"}


def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    import torch.distributed as dist

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    # a stream of our own: the context's kernels and the timing events must be
    # on the same stream (torch's default stream has handle 0, which the C ABI
    # reads as "the context's own stream")
    stream = torch.cuda.Stream(device=dev)
    assert stream.cuda_stream != 0

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    case = Case(args.workload, args.cells, args.seed)
    storage = STORAGES[args.storage]
    peak, peak_kind = read_peaks()

    main_r = measure_storage(case, storage, args, dev, stream, barrier, sample_clocks=(rank == 0))
    adjoint = measure_adjoint(dev, stream, barrier) if args.adjoint else None
    if adjoint is not None and case.n_cells:
        adjoint = {"c3_wss": adjoint, "c4_flux_split_mixed_precision": measure_c4(case, dev, stream, barrier)}
    variants = {}
    for name in [v for v in args.variants.split(",") if v and v != args.storage]:
        variants[name] = (STORAGES[name], measure_storage(case, STORAGES[name], args, dev, stream,
                                                         barrier))

    # max over ranks of every timed figure
    def vmax(vals):
        return max_over_ranks(vals, f"cuda:{dev}") if world > 1 else vals

    for r in [main_r] + [v[1] for v in variants.values()]:
        r["ms"], r["ms_e2e"], r["ms_prof"], r["lbm_ms"], r["mem_ms"] = vmax(
            [r["ms"], r["ms_e2e"], r["ms_prof"], r["lbm_ms"], r["mem_ms"]])

    if rank == 0:
        s = summarize(case, storage, main_r, args.steps, world, peak)
        traffic = read_traffic(args.workload, storage)
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            csteps, cmem, cspent = time_oracle(case, args.cpu_seconds, 10 ** 9)
            cpu = {"value": round(case.n_fluid * csteps / cspent / 1e6, 3), "unit": "MLUPS",
                   "cores": oracle_threads(), "kind": "port",
                   "sample": f"{csteps} LBM iterations ({cmem} with the membrane/IB block) of the same "
                             f"workload after 3 warm-up iterations, fp32, reference pass structure, "
                             f"{cspent:.1f} s"}
            if case.n_cells:
                cpu["membrane_node_updates_per_s"] = round(case.n_nodes * cmem / cspent, 1)
        vs = {}
        for name, (sv, r) in variants.items():
            v = summarize(case, sv, r, args.steps, world, peak)
            vs[name] = {"dtype": DTYPE_NAME[sv], "value": round(v["mlups"], 1),
                        "ms_per_step": round(v["ms_per_step"], 4),
                        "ratio_to_" + args.storage: round(v["mlups"] / s["mlups"], 3),
                        "membrane_node_updates_per_s": round(v["membrane_node_updates_per_s"], 1),
                        "e2e": round(v["mlups_e2e"], 1),
                        "k_lbm_ms": round(v["k_lbm_ms"], 5),
                        "k_lbm_frac": round(v["k_lbm_frac"], 4) if v["k_lbm_frac"] else None,
                        "membrane_block_ms": round(v["membrane_block_ms"], 4)
                        if v["membrane_block_ms"] else None,
                        "cells_removed": r["removed_end"]}
            if r["wss"] is not None and main_r["wss"] is not None:
                vs[name]["wss_rel_l2_vs_" + args.storage] = float(
                    np.linalg.norm(r["wss"] - main_r["wss"]) / np.linalg.norm(main_r["wss"]))
        bpp = lbm_bytes_per_point(storage)
        membrane = None
        if case.n_cells and main_r["blocks"]:
            nb = main_r["blocks"]
            bmn = membrane_bytes_per_node(case.nn + case.nnn)
            blk_s = s["membrane_block_ms"] * 1e-3
            membrane = {
                "block_ms": round(s["membrane_block_ms"], 4),
                "share_of_step": round(s["membrane_share"], 4),
                "stages_ms": {k: round(v / nb, 4) for k, v in main_r["stages"].items()},
                "bytes_per_node_update": round(bmn, 1),
                "node_updates_per_block": case.n_nodes,
                "achieved_gbs": round(case.n_nodes * bmn / blk_s / 1e9, 2),
                "frac": round(case.n_nodes * bmn / blk_s / 1e9 / peak, 5),
                "note": "B_mn = 72 + 36 L/N with L = 1000 footprint points per cell; the block is "
                        "latency- and atomic-bound, so it is reported as a share of the step",
            }
        result = {
            "metric": "MLUPS", "value": round(s["mlups"], 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(s["ms_per_step"], 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_NAME[storage],
            "data": "synthetic (seeded vessel geometry, wall mesh and cell placement)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "value_formula": f"fluid_points x {STAGGER} x steps / device time of the steps "
                             f"(each step {STAGGER} LBM iterations + 1 membrane/IB block)",
            "membrane_node_updates_per_s": round(s["membrane_node_updates_per_s"], 1),
            "cells_removed": main_r["removed_end"],
            "config": case.config(args.storage),
            "roofline": {"bound": "hbm", "kernel": "k_lbm",
                         "achieved": round(s["k_lbm_gbs"], 1) if s["k_lbm_gbs"] else None,
                         "peak": peak, "unit": "GB/s",
                         "frac": round(s["k_lbm_frac"], 4) if s["k_lbm_frac"] else None,
                         "traffic": None if traffic is None else round(traffic * case.n_fluid),
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_point": bpp,
                         "algorithmic_bytes_per_launch": case.n_fluid * bpp,
                         "overhead_bytes_per_point": LBM_OVERHEAD_BYTES,
                         "traffic_over_algorithmic": None if traffic is None else round(traffic / bpp, 3),
                         "k_lbm_ms_per_launch": round(s["k_lbm_ms"], 5),
                         "k_lbm_share_of_step": round(s["lbm_share"], 4) if s["lbm_share"] else None,
                         "membrane": membrane},
            "storage_variants": vs,
            "cpu_baseline": cpu,
            "e2e": {"value": round(s["mlups_e2e"], 1), "unit": "MLUPS", "h2d_bytes_per_step": 12,
                    "d2h_bytes_per_step": main_r["d2h"],
                    "copies": "per step: driving force in; FP64 mass, fp64 node positions of every "
                              "membrane and nucleus, cell status out (pinned host memory; the "
                              "positions and statuses with zf_get_cells_async, overlapping the next "
                              "step's LBM iterations, the last copy waited for inside the timed region)"},
            "adjoint": adjoint,
            "gpu_launches": main_r["launches"],
            "clocks": main_r["clocks"],
        }
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def wall_node_normals(wall):
    """Area-weighted unit normals of the wall mesh's nodes ([3][nw])."""
    xyz, tri1, nrm = wall
    t = tri1 - 1
    p = xyz.T.astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(p[t[1]] - p[t[0]], p[t[2]] - p[t[0]]), axis=1)
    acc = np.zeros((xyz.shape[1], 3))
    for v in range(3):
        np.add.at(acc, t[v], area[:, None] * nrm.T)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    return np.ascontiguousarray(acc.T, np.float32)


def run_c2(args):
    """Precision report on the workload itself (not a throughput line): the
    FP64 CPU oracle runs `--c2-steps` iterations of the reference loop; each
    storage form runs the same iterations on the GPU; the relative L2 errors of
    the fluid velocity, the density deviation, the wall shear stress and the
    membrane-node displacement are printed as one JSON line."""
    import zebraflow_b200 as zf
    case = Case(args.workload, args.cells, args.seed)
    n = args.c2_steps
    every = args.c2_avg_every
    first = n - every * ((n // 2) // every)  # the time average covers about the second half of the run
    nrm = wall_node_normals(case.wall)

    def sampled(step, wss_now):
        """Step n iterations; the mean of the WSS taken at iteration `first`
        and every `every` iterations after it (one sample per output of the
        post-processor's loop over output iterations)."""
        step(first)
        acc, k = wss_now(), 1
        for _ in range((n - first) // every):
            step(every)
            acc, k = acc + wss_now(), k + 1
        return acc / k, k

    t0 = time.perf_counter()
    lbm, oc, w = case.oracle_world("f64")
    wss_avg_ref, n_samples = sampled(w.step, lambda: w.wss(nrm)[0].astype(np.float64))
    D, U, V, W = lbm.moments()
    wss_ref, _, _ = w.wss(nrm)
    oget = oc.get()
    x_ref, live_ref = oget["x"], oget["status"] > 0
    t_oracle = time.perf_counter() - t0
    for o in (w, oc, lbm):
        o.close()
    dom = np.argwhere(case.b >= 0)
    fl = case.b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
    u_ref, rho_ref = np.stack([U, V, W])[:, fl], (D - 1.0)[fl]
    x0 = case.cells[0]

    def rel(a, b):
        ok = np.isfinite(a) & np.isfinite(b)  # wall nodes without a valid probe give no WSS
        return float(np.linalg.norm((a - b)[ok]) / np.linalg.norm(b[ok]))

    out, fields = {}, {}
    for name in ("f32", "f32dev", "f16", "bf16"):
        ctx = zf.Context(case.params(STORAGES[name]))
        ctx.set_lattice(case.b)
        ctx.set_wall(*case.wall)
        ctx.set_mesh(*case.mesh)
        ctx.set_cells(*case.cells)
        wss_avg, _ = sampled(ctx.step, lambda: ctx.wss(nrm)[0].astype(np.float64))
        wss, _, _ = ctx.wss(nrm)
        Dg, Ug, Vg, Wg = ctx.download_moments()
        x, _, status = ctx.cells()
        live = (status > 0) & live_ref  # cells alive in both runs
        u = np.stack([Ug, Vg, Wg])[:, fl]
        fields[name] = (u, (Dg - 1.0)[fl], wss, x - x0, live)
        out[name] = {"u": rel(u, u_ref), "rho_minus_1": rel((Dg - 1.0)[fl], rho_ref), "wss": rel(wss, wss_ref),
                     "wss_time_averaged": rel(wss_avg, wss_avg_ref),
                     "displacement": rel((x - x0)[:, live], (x_ref - x0)[:, live]),
                     "cells_removed": int((status <= 0).sum())}
        ctx.close()
    # each storage form against the fp32 GPU run (the storage's own effect)
    u32, r32, w32, d32, l32 = fields["f32"]
    vs32 = {}
    for name in ("f32dev", "f16", "bf16"):
        u, r, wv, dsp, live = fields[name]
        both = live & l32
        vs32[name] = {"u": rel(u, u32), "wss": rel(wv, w32), "displacement": rel(dsp[:, both], d32[:, both])}
    print(json.dumps({"report": "c2_precision_against_fp64_oracle", "workload": case.name,
                      "iterations": n, "membrane_blocks": n // 50, "fp64_oracle_seconds": round(t_oracle, 1),
                      "wss_time_average": {"first_iteration": first, "every": every, "samples": n_samples},
                      "oracle_cells_removed": int((~live_ref).sum()),
                      "relative_l2_vs_fp64_oracle": out, "relative_l2_vs_fp32_gpu": vs32}), flush=True)
    return 0


def run_sharded(args):
    """The LBM step of the workload's lattice (no cells) split into z slabs,
    one per rank, with the halo exchange after every step (strong scaling:
    the lattice is fixed, N ranks share it).  One JSON line, MLUPS of the
    whole lattice from the slowest rank's device time."""
    import torch
    import torch.distributed as dist
    import zebraflow_b200 as zf
    from zebraflow_b200 import slabs
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    nx, ny, nz, Rp, Rd, ang, g, _ = WORKLOADS[args.workload]
    b, _ = zf.gen_bifurcation(nx, ny, nz, Rp, Rd, ang)
    n_fluid = int((b > 0).sum())
    st = STORAGES[args.storage]
    slab = slabs.SlabLBM(b, world=world, rank=rank, device=local, tau=0.9, tau_from_phase=0,
                         wall_mode=zf.WALL_HALFWAY_BB, g=(0.0, 0.0, g), storage=st)
    slab.step(args.warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(local)
    e0.record(slab.stream)
    slab.step(args.steps)
    e1.record(slab.stream)
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1)
    if world > 1:
        ms = max_over_ranks([ms], f"cuda:{local}")[0]
    if rank == 0:
        print(json.dumps({"metric": "MLUPS", "value": round(n_fluid * args.steps / (ms * 1e-3) / 1e6, 1),
                          "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
                          "scaling": "strong", "dtype": DTYPE_NAME[st], "data": "synthetic",
                          "config": {"workload": args.workload + "_lbm_only", "fluid_points": n_fluid,
                                     "parallelism": f"z slabs x{world}, halo exchange every step"}}),
              flush=True)
    slab.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_split(args):
    """The coupled step (the workload's cells included) split into z slabs,
    one per rank (zebraflow_b200.slabs.SlabCoupled: the fluid sharded, the
    cells replicated, the IB coupling by owned planes with one all-reduce of
    the node velocities per membrane iteration).  Strong scaling: the workload
    is fixed, N ranks share it.  One JSON line, MLUPS of the coupled step from
    the slowest rank's device time (a step is one 50-iteration cycle)."""
    import torch
    import torch.distributed as dist
    from zebraflow_b200 import slabs
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    case = Case(args.workload, args.cells, args.seed)
    st = STORAGES[args.storage]
    p = case.params(st)
    kw = dict(tau=p.tau, tau_from_phase=0, wall_mode=WALL_HALFWAY_BB, g=tuple(p.g), storage=st,
              origin=(0.0, 0.0, 0.0), dx=DX_UM, area0=0.0, volume0=0.0)
    slab = slabs.SlabCoupled(case.b, case.wall, case.mesh, case.cells, world=world, rank=rank, device=local,
                             **kw)
    cycle = slab.stagger
    slab.step(args.warmup * cycle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(local)
    e0.record(slab.stream)
    slab.step(args.steps * cycle)
    e1.record(slab.stream)
    torch.cuda.synchronize(local)
    ms = e0.elapsed_time(e1)
    if world > 1:
        ms = max_over_ranks([ms], f"cuda:{local}")[0]
    if rank == 0:
        print(json.dumps({"metric": "MLUPS", "value": round(case.n_fluid * cycle * args.steps / (ms * 1e-3) / 1e6, 1),
                          "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
                          "scaling": "strong", "dtype": DTYPE_NAME[st], "data": "synthetic",
                          "config": {"workload": args.workload, "fluid_points": case.n_fluid,
                                     "cells": case.n_cells, "iterations_per_step": cycle,
                                     "parallelism": f"z slabs x{world}: fluid sharded, cells replicated, "
                                                    "IB by owned planes, velocity all-reduce per membrane "
                                                    "iteration"}}),
              flush=True)
    slab.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100,
                    help="timed steps; a step is one cycle of 50 LBM iterations ending in the "
                         "membrane/IB block (100 cycles = the workload's 5000 iterations)")
    ap.add_argument("--warmup", type=int, default=3, help="untimed cycles before the timed ones")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1_bifurcation_256x256x1024_2000rbc",
                    choices=sorted(WORKLOADS))
    ap.add_argument("--cells", type=int, default=None, help="override the workload's cell count")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--storage", default="f32", choices=sorted(STORAGES))
    ap.add_argument("--variants", default="f16,bf16",
                    help="comma-separated storage forms measured beside --storage")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--reference-seconds", type=float, default=90.0)
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the adjoint cost measurement on the C3 tube")
    ap.add_argument("--c2-steps", type=int, default=0,
                    help="instead of the bench line, a precision report of this many iterations "
                         "against the FP64 oracle")
    ap.add_argument("--c2-avg-every", type=int, default=50,
                    help="iterations between the WSS samples of the report's time average")
    ap.add_argument("--sharded", action="store_true",
                    help="instead of the bench line, the LBM step of the lattice split into z slabs "
                         "over the ranks (no cells)")
    ap.add_argument("--split", action="store_true",
                    help="instead of the bench line, the coupled step split into z slabs over the ranks "
                         "(fluid sharded, cells replicated)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.c2_steps > 0:
        return run_c2(args)
    if args.sharded and args.impl == "ours":
        return run_sharded(args)
    if args.split and args.impl == "ours":
        return run_split(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
