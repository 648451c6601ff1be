"""Benchmark of the resolved LBM-DEM (PSC) time step.

Default workload (dense suspension, seeded synthetic input): 256^3 D3Q19
lattice, periodic in x, y and z; 2000 spheres with diameters uniform in
[8, 12] lattice units placed by random sequential addition (1 lu gap);
Gaussian velocities (sigma 1e-3); density ratio 2.0; Hertz-Mindlin contacts
(E=1e5, nu=0.3, restitution 0.9, friction 0.3); uniform body force 1e-6 (x) on
fluid and particles; tau=0.6 with Smagorinsky Cs=0.1 (reference lagged form);
DEM sub-cycled 10x per lattice step.  A step = map particles -> fused PSC
collide-stream with force reduction -> 10 DEM sub-steps.  `value` times the
product's PSCLattice3D.run(), which pipelines the steps where that is faster
(the x-blocks no particle can reach are stepped while the DEM and the next map
run on a second stream; identical results; `pipelined` says which form ran);
`sequential` and `phases_ms` time the plain collide/stream/DEM loop, and the
roofline is the fused step kernel's.  --no-pipeline times the plain loop as
`value`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|f16|bf16]
    python bench.py --workload c5        # 512x512x256 channel, 20000 spheres, LES
    python bench.py --workload c1        # single sphere settling, 64x64x128
    python bench.py --workload pdrop     # packed-bed pressure drop, 722x242x242, open boundaries
    python bench.py --impl reference     # FP64 CPU restatement of the reference path
    python bench.py --adjoint [--adjoint-fd K]   # drag gradient on the frozen-bed channel (below)

Prints ONE JSON line (rank 0).  Multi-GPU: independent replicas (the path is
one GPU per the workload definition), aggregate throughput, weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS & HBM-roofline % for D3Q19 PSC step, FP16-store vs FP32 at ≤1e-3 drag err"
BYTES_PER_CELL = {"f32": 152, "f16": 76, "bf16": 76}   # 19 reads + 19 writes of the storage type
# DRAM read + write per cell of the step kernel, from the ncu capture of the
# 128^3 case (see profiles/k_psc_step_128cube_full.md), scaled by the cells of a launch
TRAFFIC_PER_CELL = {"f32": 175.7, "f16": 85.2, "bf16": 85.2}

# Workloads (lattice units).  c2 is the headline configuration; c5 and c1 are
# the large channel and the single settling sphere.  Parameters the workload
# descriptions leave open are fixed here and used identically by the oracle.
WORKLOADS = {
    "c2": dict(desc="dense suspension 256^3 periodic, 2000 spheres d~U[8,12], Hertz e=0.9, body force 1e-6, "
                    "tau=0.6, Smagorinsky Cs=0.1 (lagged), 10 DEM sub-steps",
               shape=(256, 256, 256), n=2000, dmin=8.0, dmax=12.0, gap=1.0, walls_z=False, tau=0.6, cs=0.1,
               fluid_force=(1e-6, 0.0, 0.0), gravity=(1e-6, 0.0, 0.0), rho_p=2.0, vel_sigma=1e-3, sub=10),
    "c5": dict(desc="large channel 512x512x256, periodic x/y, no-slip walls at z=0,255, 20000 spheres "
                    "d~U[6,10], Hertz e=0.9, body force 1e-6, tau=0.51, Smagorinsky Cs=0.12 (lagged), "
                    "10 DEM sub-steps",
               shape=(512, 512, 256), n=20000, dmin=6.0, dmax=10.0, gap=0.5, walls_z=True, tau=0.51, cs=0.12,
               fluid_force=(1e-6, 0.0, 0.0), gravity=(1e-6, 0.0, 0.0), rho_p=2.0, vel_sigma=1e-3, sub=10),
    "c1": dict(desc="single sphere d=12 settling in 64x64x128, periodic x/y, no-slip walls at z=0,127, density "
                    "ratio 2.5, gravity 1e-5 (-z, buoyancy-reduced on the particle), tau=0.6, Smagorinsky Cs=0.1 "
                    "(lagged), Hertz with the bottom wall, 10 DEM sub-steps",
               shape=(64, 64, 128), n=1, dmin=12.0, dmax=12.0, gap=0.0, walls_z=True, tau=0.6, cs=0.1,
               fluid_force=None, gravity=(0.0, 0.0, -1e-5 * (1.0 - 1.0 / 2.5)), rho_p=2.5, vel_sigma=0.0, sub=10),
    # the packed-bed pressure-drop driver's configuration (pressure_drop_fully.py:106-116, 120-170, 200-245):
    # 30 x 10 x 10 particle diameters at 24 cells per diameter, tau 0.68, Re 0.8 (inlet 2.0e-3 lu), frozen
    # bed, linear contacts, one DEM sub-step, Ladd velocity inlet at x = 0, Zou-He pressure (rho = 1) at
    # x = Nx-1, periodic y / z; the bed is seeded random sequential addition (the driver reads a packing file)
    "pdrop": dict(desc="packed-bed pressure drop 722x242x242, Ladd velocity inlet 2.0e-3 at x=0, Zou-He pressure "
                       "outlet rho=1 at x=Nx-1, periodic y/z, 1500 frozen spheres d=24 (RSA, 24 lu clear of the "
                       "inlet and outlet), tau=0.68, Smagorinsky off, linear contacts, 1 DEM sub-step",
                  shape=(722, 242, 242), n=1500, dmin=24.0, dmax=24.0, gap=0.5, walls_z=False, tau=0.68, cs=None,
                  fluid_force=None, gravity=(0.0, 0.0, 0.0), rho_p=2.5, vel_sigma=0.0, sub=1, u_in=2.0e-3,
                  x_clear=24.0),
}
W = dict(WORKLOADS["c2"], key="c2")
NX, NY, NZ = W["shape"]
NP = W["n"]
SUB = W["sub"]
TAU = W["tau"]
CS = W["cs"]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(seed=2024):
    """Seeded inputs of the selected workload (lattice units)."""
    from tests.gpu_util import rsa_spheres_grid   # pure numpy helper
    rng = np.random.default_rng(seed)
    if W["key"] == "c1":
        pos = np.array([[NX / 2 + rng.uniform(-0.5, 0.5), NY / 2 + rng.uniform(-0.5, 0.5), NZ - 18.0]])
        rad = np.array([0.5 * W["dmin"]])
    elif "u_in" in W:
        xc = W["x_clear"]
        pos, rad = rsa_spheres_grid(rng, NP, (NX - 2 * xc, NY, NZ), W["dmin"], W["dmax"], gap=W["gap"], margin=0.5)
        pos[:, 0] += xc
    else:
        zlo = 1.0 if W["walls_z"] else None
        zhi = NZ - 1.0 if W["walls_z"] else None
        pos, rad = rsa_spheres_grid(rng, NP, (NX, NY, NZ), W["dmin"], W["dmax"], gap=W["gap"], zmin=zlo, zmax=zhi,
                                    margin=0.5)
    vel = rng.normal(0.0, W["vel_sigma"], (NP, 3)) if W["vel_sigma"] > 0 else np.zeros((NP, 3))
    mass = W["rho_p"] * 4.0 / 3.0 * np.pi * rad ** 3
    return pos, rad, vel, mass


def cell_types():
    ct = np.full((NX, NY, NZ), 1, np.int32)
    if W["walls_z"]:
        ct[:, :, 0] = ct[:, :, -1] = 8
    if "u_in" in W:
        ct[0] = 262144 | 8192     # VEL_INLET_LADD | LEFT
        ct[-1] = 256 | 4096       # Pre_ZOUHE | RIGHT
    return ct


def open_presets(vel, rho):
    """Inlet velocity and outlet density of the open-boundary workload (in place)."""
    vel[0, ..., 0] = W["u_in"]
    rho[-1] = 1.0


def build_gpu(storage, pos, rad, vel, mass):
    from lbdem_taichi_b200 import Vector3
    from lbdem_taichi_b200.dem3d.demconfig import (DEMSolverConfig, DomainBounds, HertzContactConfig,
                                                   LinearContactConfig)
    from lbdem_taichi_b200.dem3d.demsolver import DEMSolver
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    domain = (0.0, float(NX), 0.0, float(NY), 0.0, float(NZ))
    opened = "u_in" in W
    contact = (LinearContactConfig(stiffness_normal=4.5e3, stiffness_tangential=2.5e3, damping_normal=0.3,
                                   damping_tangential=0.2, pp_friction=0.15, pw_friction=0.15) if opened else
               HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9))
    cfg = DEMSolverConfig(DomainBounds(*domain), 1.0 / SUB, Vector3(*W["gravity"]), contact)
    cfg.set_particle_properties(elastic_modulus=1e5, poisson_ratio=0.3, max_coordinate_number=16)
    cfg.set_wall_properties(elastic_modulus=1e5, poisson_ratio=0.3)
    cfg.set_periodic_boundaries(not opened, True, not W["walls_z"])
    dem = DEMSolver(cfg)
    dem.init_particle_arrays(rad, mass, pos, vel, Vector3(0, 0, 0), Vector3(NX, NY, NZ))
    dem.set_contact_model("linear" if opened else "hertz")
    if opened:
        dem.gf.freeze.from_numpy(np.ones(len(rad), np.int32))
    lat = PSCLattice3D(NX, NY, NZ, 1.0 / TAU, 1.0, 1.0, 1.0, dem, smagorinsky="off" if CS is None else "reference",
                       body_force=W["fluid_force"], storage=storage)
    if CS is not None:
        lat.SmagorinskyConstant = CS
    if W["walls_z"] or opened:
        lat.CT.from_numpy(cell_types())
    if opened:
        v, r = lat.vel.to_numpy(), lat.rho.to_numpy()
        open_presets(v, r)
        lat.vel.from_numpy(v)
        lat.rho.from_numpy(r)
    lat.initialize()
    return lat, dem


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, index):
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
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                p = [s.strip() for s in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                   p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, world, device="cuda"):
    """The slowest rank's value of x (a time in ms).  Every rank calls it, in
    the same order, for every reduced quantity."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world, cells, steps, ms):
    """Whole-job MLUPS of `world` replicas that each updated `cells` cells
    `steps` times, timed by the slowest rank (ms)."""
    return world * cells * steps / (ms * 1e-3) / 1e6


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from lbdem_taichi_b200 import _native as Nat

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    pos, rad, vel, mass = workload()
    lat, dem = build_gpu(args.storage, pos, rad, vel, mass)
    st = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        lat.step(SUB)
    torch.cuda.synchronize()
    lat.check_status()
    dem.check_status()

    # ---- device-resident throughput (inputs already in HBM).  When the
    # populations do not exceed L2 several times over, a 256 MB buffer is
    # rewritten between steps (outside the per-step events) to flush L2.
    cells = NX * NY * NZ
    pop_gb = 2 * 19 * cells * (4 if args.storage == "f32" else 2) / 1e9
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda") if pop_gb <= 0.5 else None
    mk = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ev_step = [(mk(), mk()) for _ in range(args.steps)]
    ev_phase = [(mk(), mk(), mk()) for _ in range(args.steps)]   # before map, after step kernel, after DEM
    lat._kernel_events = []
    Nat.reset_launch_count()
    barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    cpu0 = time.perf_counter()
    with Clocks(local) as clk:
        t0.record(st)
        for k in range(args.steps):
            if flush is not None:
                flush.fill_(float(k))
            lat._kernel_events = ev_step[k]
            ev_phase[k][0].record(st)
            lat.collide()
            lat.stream()
            ev_phase[k][1].record(st)
            dem.run_substeps(SUB)
            ev_phase[k][2].record(st)
        t1.record(st)
        cpu_launch_ms = (time.perf_counter() - cpu0) * 1e3 / args.steps
        torch.cuda.synchronize()
    lat._kernel_events = None
    launches = Nat.launch_count()
    barrier()
    # with a flush the step time is the sum of the per-step events (map to end of DEM)
    ms = t0.elapsed_time(t1) if flush is None else sum(a.elapsed_time(c) for a, _, c in ev_phase)
    ms_seq = ms
    # ---- the product's run(): the sequential loop above, pipelined (the blocks
    # no particle can reach are stepped while the DEM and the next map run on a
    # second stream).  Needs inputs larger than L2 (no flush between steps).
    pipelined = flush is None and not args.no_pipeline
    if pipelined:
        lat.run(40, SUB)          # run()'s automatic choice is measured here, outside the timed region
        pipelined = bool(lat._pipeline_choice)
        torch.cuda.synchronize()
        Nat.reset_launch_count()
        barrier()
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            t0.record(st)
            cpu0 = time.perf_counter()
            lat.run(args.steps, SUB)
            t1.record(st)
            cpu_launch_ms = (time.perf_counter() - cpu0) * 1e3 / args.steps
            torch.cuda.synchronize()
        launches = Nat.launch_count()
        barrier()
        ms = t0.elapsed_time(t1)
    ms = max_over_ranks(ms, world)
    ms_seq = max_over_ranks(ms_seq, world)
    kern_ms = statistics.mean(a.elapsed_time(b) for a, b in ev_step)
    lbm_ms = statistics.mean(a.elapsed_time(b) for a, b, _ in ev_phase)
    dem_ms = statistics.mean(b.elapsed_time(c) for _, b, c in ev_phase)
    lat.check_status()
    dem.check_status()
    clocks = clk.summary()

    # ---- end to end through the public API with host buffers: every step
    # uploads the particle state from pinned host memory and reads back the
    # per-particle fluid force/torque and the new state
    h_in = torch.empty((2, NP, 3), dtype=torch.float64).pin_memory()
    h_out = torch.empty((4, NP, 3), dtype=torch.float64).pin_memory()
    h_in[0].copy_(dem._t["position"])
    h_in[1].copy_(dem._t["velocity"])
    torch.cuda.synchronize()
    e_steps = max(1, args.steps // 2)
    barrier()
    tw0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(e_steps):
        dem._t["position"].copy_(h_in[0], non_blocking=True)
        dem._t["velocity"].copy_(h_in[1], non_blocking=True)
        dem._touched("position")
        lat.step(SUB)
        h_out[0].copy_(dem._t["force_fluid"], non_blocking=True)
        h_out[1].copy_(dem._t["moment_fluid"], non_blocking=True)
        h_out[2].copy_(dem._t["position"], non_blocking=True)
        h_out[3].copy_(dem._t["velocity"], non_blocking=True)
        st.synchronize()
        h_in[0].copy_(h_out[2])
        h_in[1].copy_(h_out[3])
    e1.record(st)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - tw0) * 1e3)
    e2e_ms = max_over_ranks(e2e_ms, world)

    value = job_mlups(world, cells, args.steps, ms)
    e2e_value = job_mlups(world, cells, e_steps, e2e_ms)
    peak, peak_kind = peaks()
    bpc = BYTES_PER_CELL[args.storage]
    l2_note = (f"inputs larger than L2 (populations {pop_gb:.2f} GB); no flush" if flush is None else
               f"populations {pop_gb:.2f} GB; L2 flushed between steps (256 MB rewrite outside the step events)")
    achieved = bpc * cells / (kern_ms * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": {"workload": W["desc"], "name": W["key"],
                   "lattice": [NX, NY, NZ], "particles": NP, "dem_subcycles": SUB, "storage": args.storage,
                   "l2": l2_note, "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "kernel": f"lbdem_psc_step_{args.storage}", "kernel_ms": round(kern_ms, 4),
                     "bytes_per_cell": bpc,
                     "traffic": round(TRAFFIC_PER_CELL[args.storage] * cells / 1e9, 4),
                     "traffic_unit": "GB per launch (DRAM read+write per cell from the 128^3 ncu capture x cells)"},
        "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 2 * NP * 3 * 8,
                "d2h_bytes_per_step": 4 * NP * 3 * 8},
        "gpu_launches": launches,
        "pipelined": pipelined,
        "pipeline_probe_ms": [round(v, 4) for v in lat._pipeline_probe] if lat._pipeline_probe else None,
        "sequential": {"value": round(job_mlups(world, cells, args.steps, ms_seq), 2),
                       "ms_per_step": round(ms_seq / args.steps, 4)},
        "phases_ms": {"map+step": round(lbm_ms, 4), "step_kernel": round(kern_ms, 4), f"dem_{SUB}_substeps": round(dem_ms, 4),
                      "host_launch_per_step": round(cpu_launch_ms, 4)},
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(pos, rad, vel, mass, budget_s=args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def slab_depth():
    """z-depth of the CPU sample: the oracle maps by probing every particle for
    every cell, so the slab keeps cells x particles near 2e8 per step."""
    return int(max(1, min(NZ, 8, 2e8 // max(1, NX * NY * NP))))


def cpu_sample(pos, rad, vel, mass, nz_slab):
    """Oracle (FP64 C restatement of the reference) on a z-slab of the workload
    carrying every particle: same per-cell work (grains2lattice probes all
    particles for every cell), NX x NY x `nz_slab` cells."""
    from oracle.oracle import OracleDEM, OracleGrains, OracleLattice
    lat = OracleLattice(NX, NY, nz_slab, 1.0 / TAU, smag=CS is not None, psc=True, force=W["fluid_force"],
                        smag_cs=CS if CS is not None else 0.1)
    lat.ct[...] = cell_types()[:, :, :nz_slab]
    if "u_in" in W:
        open_presets(lat.vel, lat.rho)
    dem = OracleDEM(pos, vel, rad, mass, dt=1.0 / SUB, gravity=W["gravity"], domain=(0, NX, 0, NY, 0, NZ),
                    periodic=(True, True, not W["walls_z"]), E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3, pp_mu=0.3,
                    pw_mu=0.3, pp_e=0.9, pw_e=0.9, max_coord=16)
    g = OracleGrains(dem.pos, dem.radius, dem.vel, dem.omega)
    g.force_fluid, g.moment_fluid = dem.force_fluid, dem.moment_fluid
    lat.initialize()
    return lat, dem, g


def cpu_step(lat, dem, g):
    lat.grains2lattice(g)
    lat.collide()
    lat.lattice2grains(g)
    lat.stream()
    for _ in range(SUB):
        dem.run_simulation()


def cpu_baseline(pos, rad, vel, mass, budget_s=20.0):
    nz_slab = slab_depth()
    lat, dem, g = cpu_sample(pos, rad, vel, mass, nz_slab)
    t0 = time.perf_counter()
    steps = 0
    while True:
        cpu_step(lat, dem, g)
        steps += 1
        if time.perf_counter() - t0 > budget_s * 0.5 or steps >= 50:
            break
    dt = time.perf_counter() - t0
    cells = NX * NY * nz_slab
    return {"value": round(cells * steps / dt / 1e6, 4), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{steps} full steps (map, collide, force reduction, stream, {SUB} DEM sub-steps) on a "
                      f"{NX}x{NY}x{nz_slab} slab of the workload carrying all {NP} particles; FP64 C "
                      f"restatement, OpenMP {os.cpu_count()} threads"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pos, rad, vel, mass = workload()
    nz_slab = slab_depth()
    lat, dem, g = cpu_sample(pos, rad, vel, mass, nz_slab)
    for _ in range(args.warmup_ref):
        cpu_step(lat, dem, g)
    t0 = time.perf_counter()
    for _ in range(args.steps_ref):
        cpu_step(lat, dem, g)
    dt = time.perf_counter() - t0
    cells = NX * NY * nz_slab
    v = cells * args.steps_ref / dt / 1e6
    sample = f"{NX}x{NY}x{nz_slab} slab of the workload with all {NP} particles per step"
    # the GPU arm's config; the reference computes in FP64 on the host cores (no GPU)
    out = {"metric": METRIC, "value": round(v, 4), "unit": "MLUPS", "impl": "reference", "n_gpus": args.gpus,
           "device": "cpu", "steps": args.steps_ref, "warmup": args.warmup_ref,
           "ms_per_step": round(dt * 1e3 / args.steps_ref, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": W["desc"], "name": W["key"], "lattice": [NX, NY, NZ], "particles": NP,
                      "dem_subcycles": SUB, "storage": "f64", "sample": f"per step: {sample}",
                      "parallelism": f"{os.cpu_count()} host threads"},
           "cpu_baseline": {"value": round(v, 4), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(v, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# Differentiation workload: 128^3 channel (OBSTACLE walls at z = 0 and 127,
# periodic x/y), 500 frozen spheres of diameter 10 placed by seeded random
# sequential addition in z < 64 (0.2 lu gap), body force g_x = 2e-6, tau 0.6,
# Smagorinsky off, FP32, smooth solid fraction; loss = total x-drag on the bed
# after step 500; gradient w.r.t. g_x and every sphere centre by the adjoint
# with checkpoints every 50 steps.  --adjoint-fd K adds FP64 central finite
# differences (h = 1e-4 relative) of the oracle's forward for g_x and the K-1
# largest position components.
# ---------------------------------------------------------------------------
ADJ_N, ADJ_NP, ADJ_STEPS, ADJ_EVERY, ADJ_G = 128, 500, 500, 50, 2e-6


def adjoint_workload(seed=2024):
    from tests.gpu_util import rsa_spheres
    rng = np.random.default_rng(seed)
    pos, rad = rsa_spheres(rng, ADJ_NP, (ADJ_N, ADJ_N, ADJ_N), 10.0, 10.0, gap=0.2, zmax=ADJ_N / 2, margin=1.0)
    ct = np.full((ADJ_N,) * 3, 1, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = 8
    return pos, rad, ct


def run_adjoint(args):
    import torch

    from lbdem_taichi_b200 import _native as Nat
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from lbdem_taichi_b200.lbdem.adjoint import FrozenBedDrag
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    from tests.gpu_util import make_dem
    pos, rad, ct = adjoint_workload()
    n = len(rad)
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    dem = make_dem((0.0, ADJ_N, 0.0, ADJ_N, 0.0, ADJ_N), 0.1, (0, 0, 0),
                   HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9),
                   rad, mass, pos, np.zeros((n, 3)), periodic=(True, True, False), freeze=np.ones(n, np.int32))
    lat = PSCLattice3D(ADJ_N, ADJ_N, ADJ_N, 1.0 / TAU, 1.0, 1.0, 1.0, dem, body_force=(ADJ_G, 0.0, 0.0),
                       solid_fraction="smooth")
    lat.CT.from_numpy(ct)
    prob = FrozenBedDrag(lat, ADJ_STEPS, direction=(1.0, 0.0, 0.0), checkpoint_every=ADJ_EVERY)
    prob.forward()
    prob.backward()
    reps = max(1, min(args.steps, 5))
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    fwd, bwd = [], []
    Nat.reset_launch_count()
    for _ in range(reps):
        torch.cuda.synchronize()
        e0.record()
        L = prob.forward()
        e1.record()
        gF, gP = prob.backward()
        e2.record()
        torch.cuda.synchronize()
        fwd.append(e0.elapsed_time(e1))
        bwd.append(e1.elapsed_time(e2))
    launches = Nat.launch_count() // reps
    cells = ADJ_N ** 3
    out = {"metric": "C4 drag gradient: forward + adjoint wall time (checkpointed)", "value": round(
        statistics.median(fwd) + statistics.median(bwd), 2), "unit": "ms", "higher_is_better": False,
        "n_gpus": 1, "steps": ADJ_STEPS, "reps": reps, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "128^3 channel, 500 frozen spheres d=10 (RSA, z<64), g_x=2e-6, tau=0.6, "
                               "500 steps, checkpoints every 50, smooth solid fraction"},
        "forward_ms": round(statistics.median(fwd), 2), "backward_ms": round(statistics.median(bwd), 2),
        "forward_mlups": round(cells * ADJ_STEPS / statistics.median(fwd) / 1e3, 1),
        "gpu_launches": launches, "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 2),
        "loss": L, "dL_dgx": float(gF[0]), "dL_dpos_absmax": float(np.abs(gP).max())}
    if args.adjoint_fd > 0:
        from oracle.oracle import frozen_bed_drag
        F = np.array([ADJ_G, 0.0, 0.0])
        shape = (ADJ_N,) * 3

        def L64(Fv, P):
            return frozen_bed_drag(shape, 1.0 / TAU, ct, rad, P, Fv, ADJ_STEPS)
        t0 = time.perf_counter()
        checks = []
        h = 1e-4 * ADJ_G
        fd = (L64(F + [h, 0, 0], pos) - L64(F - [h, 0, 0], pos)) / (2 * h)
        checks.append({"param": "g_x", "adjoint": float(gF[0]), "fd64": fd, "rel": abs(gF[0] - fd) / abs(fd)})
        order = np.argsort(-np.abs(gP).ravel())[: args.adjoint_fd - 1]
        for flat in order:
            i, k = divmod(int(flat), 3)
            hp = 1e-4 * abs(pos[i, k])
            pp, pm = pos.copy(), pos.copy()
            pp[i, k] += hp
            pm[i, k] -= hp
            fdp = (L64(F, pp) - L64(F, pm)) / (2 * hp)
            checks.append({"param": f"pos[{i},{'xyz'[k]}]", "adjoint": float(gP[i, k]), "fd64": fdp,
                           "rel": abs(gP[i, k] - fdp) / abs(fdp)})
        out["fd_check"] = {"h": "1e-4 relative, central, FP64 oracle forward", "cpu_seconds":
                           round(time.perf_counter() - t0, 1), "cores": os.cpu_count(), "params": checks,
                           "max_rel": max(c["rel"] for c in checks)}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pipeline", action="store_true", help="time the sequential loop (collide, stream, DEM)")
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--size", type=int, default=0, help="cube edge override; only for small profiling cases")
    ap.add_argument("--particles", type=int, default=0, help="particle count override; only for profiling")
    ap.add_argument("--adjoint", action="store_true", help="drag-gradient workload instead of the step")
    ap.add_argument("--adjoint-fd", type=int, default=0, help="FP64 finite-difference checks (count)")
    args = ap.parse_args()
    global W, NX, NY, NZ, NP, SUB, TAU, CS
    W = dict(WORKLOADS[args.workload], key=args.workload)
    NX, NY, NZ = W["shape"]
    NP, SUB, TAU, CS = W["n"], W["sub"], W["tau"], W["cs"]
    if args.size:
        NX = NY = NZ = args.size
    if args.particles:
        NP = args.particles
    if args.adjoint:
        run_adjoint(args)
        return
    args.steps_ref = max(1, min(args.steps, 3))
    args.warmup_ref = 1
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
