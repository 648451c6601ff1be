"""Benchmark of the resolved LBM-DEM (PSC) time step.

Workload (dense suspension, seeded synthetic input): 256^3 D3Q19 lattice,
periodic in x, y and z; 2000 spheres with diameters uniform in [8, 12] lattice
units placed by random sequential addition (1 lu gap); Gaussian velocities
(sigma 1e-3); density ratio 2.0; Hertz-Mindlin contacts (E=1e5, nu=0.3,
restitution 0.9, friction 0.3); uniform body force 1e-6 (x) on fluid and
particles; tau=0.6 with Smagorinsky Cs=0.1 (reference lagged form); DEM
sub-cycled 10x per lattice step.  A step = map particles -> fused PSC
collide-stream with force reduction -> 10 DEM sub-steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|f16|bf16]
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
NX = NY = NZ = 256
NP = 2000       # overridable (--size/--particles) only for small profiling cases
SUB = 10
TAU = 0.6
CS = 0.1
GBODY = 1e-6
BYTES_PER_CELL = {"f32": 152, "f16": 76, "bf16": 76}   # 19 reads + 19 writes of the storage type


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(seed=2024):
    """Seeded C2 inputs (lattice units)."""
    from tests.gpu_util import rsa_spheres   # pure numpy helper
    rng = np.random.default_rng(seed)
    pos, rad = rsa_spheres(rng, NP, (NX, NY, NZ), 8.0, 12.0, gap=1.0, margin=0.5)
    vel = rng.normal(0.0, 1e-3, (NP, 3))
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    return pos, rad, vel, mass


def build_gpu(storage, pos, rad, vel, mass):
    from lbdem_taichi_b200 import Vector3
    from lbdem_taichi_b200.dem3d.demconfig import DEMSolverConfig, DomainBounds, HertzContactConfig
    from lbdem_taichi_b200.dem3d.demsolver import DEMSolver
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    domain = (0.0, float(NX), 0.0, float(NY), 0.0, float(NZ))
    cfg = DEMSolverConfig(DomainBounds(*domain), 1.0 / SUB, Vector3(GBODY, 0, 0),
                          HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9))
    cfg.set_particle_properties(elastic_modulus=1e5, poisson_ratio=0.3, max_coordinate_number=16)
    cfg.set_wall_properties(elastic_modulus=1e5, poisson_ratio=0.3)
    cfg.set_periodic_boundaries(True, True, True)
    dem = DEMSolver(cfg)
    dem.init_particle_arrays(rad, mass, pos, vel, Vector3(0, 0, 0), Vector3(NX, NY, NZ))
    dem.set_contact_model("hertz")
    lat = PSCLattice3D(NX, NY, NZ, 1.0 / TAU, 1.0, 1.0, 1.0, dem, smagorinsky="reference",
                       body_force=(GBODY, 0.0, 0.0), storage=storage)
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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

    # ---- device-resident throughput (inputs already in HBM); the populations
    # (1.27 GB FP32) exceed L2, so no flush is needed between steps
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
    ms = t0.elapsed_time(t1)
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
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
    e2e_t = torch.tensor([e2e_ms], device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_ms = float(e2e_t.item())

    cells = NX * NY * NZ
    value = world * cells * args.steps / (ms * 1e-3) / 1e6
    e2e_value = world * cells * e_steps / (e2e_ms * 1e-3) / 1e6
    peak, peak_kind = peaks()
    bpc = BYTES_PER_CELL[args.storage]
    achieved = bpc * cells / (kern_ms * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": {"workload": "dense suspension 256^3 periodic, 2000 spheres d~U[8,12], Hertz e=0.9, "
                               "body force 1e-6, tau=0.6, Smagorinsky Cs=0.1 (lagged), 10 DEM sub-steps",
                   "lattice": [NX, NY, NZ], "particles": NP, "dem_subcycles": SUB, "storage": args.storage,
                   "l2": "inputs larger than L2 (populations 1.27 GB FP32 / 0.64 GB 16-bit); no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "kernel": f"lbdem_psc_step_{args.storage}", "kernel_ms": round(kern_ms, 4),
                     "bytes_per_cell": bpc, "traffic": None},
        "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 2 * NP * 3 * 8,
                "d2h_bytes_per_step": 4 * NP * 3 * 8},
        "gpu_launches": launches,
        "phases_ms": {"map+step": round(lbm_ms, 4), "step_kernel": round(kern_ms, 4), "dem_10_substeps": round(dem_ms, 4),
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


def cpu_sample(pos, rad, vel, mass, nz_slab=8):
    """Oracle (FP64 C restatement of the reference) on a z-slab of the workload
    carrying every particle: same per-cell work (grains2lattice probes all
    particles for every cell), 256x256x`nz_slab` cells."""
    from oracle.oracle import OracleDEM, OracleGrains, OracleLattice
    lat = OracleLattice(NX, NY, nz_slab, 1.0 / TAU, smag=True, psc=True, force=(GBODY, 0.0, 0.0),
                        smag_cs=CS)
    dem = OracleDEM(pos, vel, rad, mass, dt=1.0 / SUB, gravity=(GBODY, 0, 0), domain=(0, NX, 0, NY, 0, NZ),
                    periodic=(True, True, True), E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3, pp_mu=0.3, pw_mu=0.3,
                    pp_e=0.9, pw_e=0.9, max_coord=16)
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
    nz_slab = 8
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
            "sample": f"{steps} full steps (map, collide, force reduction, stream, 10 DEM sub-steps) on a "
                      f"{NX}x{NY}x{nz_slab} slab of the workload carrying all {NP} particles; FP64 C "
                      f"restatement, OpenMP {os.cpu_count()} threads"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pos, rad, vel, mass = workload()
    lat, dem, g = cpu_sample(pos, rad, vel, mass)
    for _ in range(args.warmup_ref):
        cpu_step(lat, dem, g)
    t0 = time.perf_counter()
    for _ in range(args.steps_ref):
        cpu_step(lat, dem, g)
    dt = time.perf_counter() - t0
    cells = NX * NY * 8
    v = cells * args.steps_ref / dt / 1e6
    out = {"metric": METRIC, "value": round(v, 4), "unit": "MLUPS", "impl": "reference", "n_gpus": 0,
           "steps": args.steps_ref, "warmup": args.warmup_ref, "ms_per_step": round(dt * 1e3 / args.steps_ref, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "dense suspension 256^3 periodic, 2000 spheres d~U[8,12] (per-step sample: "
                                  "256x256x8 slab with all particles)"},
           "cpu_baseline": {"value": round(v, 4), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                            "sample": "256x256x8 slab of the workload with all 2000 particles per step"},
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
    ap.add_argument("--size", type=int, default=256, help="cube edge; non-default only for profiling")
    ap.add_argument("--particles", type=int, default=2000, help="non-default only for profiling")
    ap.add_argument("--adjoint", action="store_true", help="drag-gradient workload instead of the step")
    ap.add_argument("--adjoint-fd", type=int, default=0, help="FP64 finite-difference checks (count)")
    args = ap.parse_args()
    if args.adjoint:
        run_adjoint(args)
        return
    global NX, NY, NZ, NP
    NX = NY = NZ = args.size
    NP = args.particles
    args.steps_ref = max(1, min(args.steps, 3))
    args.warmup_ref = 1
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
