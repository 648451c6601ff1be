"""Benchmark of the resolved LBM-DEM (PSC) time step.

Default workload (dense suspension, seeded synthetic input; ``cases.py``):
256^3 D3Q19 lattice, periodic in x, y and z; 2000 spheres with diameters
uniform in [8, 12] lattice units placed by random sequential addition (1 lu
gap); Gaussian velocities (sigma 1e-3); density ratio 2.0; Hertz-Mindlin
contacts (E=1e5, nu=0.3, restitution 0.9, friction 0.3); uniform body force
1e-6 (x) on fluid and particles; tau=0.6 with Smagorinsky Cs=0.1 (reference
lagged form); DEM sub-cycled 10x per lattice step.  A step = map particles ->
fused PSC collide-stream with force reduction -> 10 DEM sub-steps.

`value` times the product's PSCLattice3D.run(), which pipelines the steps where
that is faster (the x-blocks no particle can reach are stepped while the DEM
and the next map run on a second stream; identical results; `pipelined` says
which form ran); `sequential` and `phases_ms` time the plain collide/stream/DEM
loop, and the roofline is the fused step kernel's.  --no-pipeline times the
plain loop as `value`.  `storage_forms` repeats the measurement for FP32, FP16
and BF16 population storage in the same process (the metric's two arms side by
side) with each form's speed-ups over FP32 and, for the full-size dense
suspension, its per-step drag error against the FP64 record of the same run
(tests/golden/c2_fp64.npz, written by tests/golden/make_fullsize.py).

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
from contextlib import contextmanager

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lbdem_taichi_b200 import cases  # noqa: E402

METRIC = "MLUPS & HBM-roofline % for D3Q19 PSC step, FP16-store vs FP32 at ≤1e-3 drag err"
# storage forms: population storage, and "f32-lag16" = FP32 populations with
# the lagged Smagorinsky state in FP16 (cases.split_form)
FORMS = ("f32", "f16", "bf16", "f32-lag16")
BYTES_PER_CELL = {"f32": 152, "f16": 76, "bf16": 76, "f32-lag16": 152}   # 19 reads + 19 writes of the storage type
# DRAM read + write per cell of one step-kernel launch: ncu dram__bytes_read.sum
# + dram__bytes_write.sum of a launch on the 192^3 dense suspension (844
# spheres, the same solid fraction), divided by its cells; populations 1.08 GB
# (FP32) / 0.54 GB (16-bit), both beyond the 126 MB L2
TRAFFIC_PER_CELL = {"f32": 188.4, "f16": 98.9, "bf16": 98.0, "f32-lag16": 169.0}
FIXTURE = os.path.join(ROOT, "tests", "golden", "c2_fp64.npz")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed regions
# ---------------------------------------------------------------------------
_SAMPLER = r"""
import sys, time
try:
    import pynvml as N
    N.nvmlInit()
    key = sys.argv[1]
    h = N.nvmlDeviceGetHandleByUUID(key) if key.startswith("GPU-") else N.nvmlDeviceGetHandleByIndex(int(key))
    mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
except Exception as e:
    open(sys.argv[2], "w").write("error %s\n" % e)
    sys.exit(0)
out = open(sys.argv[2], "w", buffering=1)
out.write("max %d\n" % mx)
while True:
    t = time.time()
    out.write("%.6f %d %d\n" % (t, N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM),
                                N.nvmlDeviceGetCurrentClocksEventReasons(h)))
    time.sleep(0.002)
"""
_REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
            0x80: "hw_power_brake_slowdown"}


class Clocks:
    """SM clock and throttle reasons read through NVML every ~2 ms by a child
    process (it shares no interpreter lock with the launching thread), from
    before the warm-up to the end of the bench; summary() keeps the samples
    that fall inside the timed windows."""

    def __init__(self, device):
        self.key = self._nvml_key(device)
        fd, self.path = tempfile.mkstemp(suffix=".clk")
        os.close(fd)
        self.windows = []
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _SAMPLER, self.key, self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    @staticmethod
    def _nvml_key(device):
        import torch
        try:
            return "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [v for v in vis.split(",") if v.strip()]
            return ids[device].strip() if device < len(ids) and ids[device].strip().isdigit() else str(device)

    def wait_ready(self, timeout=15.0):
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout:
            with open(self.path) as fh:
                if len(fh.readlines()) >= 2:
                    return
            time.sleep(0.05)

    @contextmanager
    def window(self):
        t0 = time.time()
        yield
        self.windows.append((t0, time.time()))

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.stop()
        lines = open(self.path).read().splitlines() if os.path.exists(self.path) else []
        os.remove(self.path)
        mx, rows = None, []
        for ln in lines:
            p = ln.split()
            if p and p[0] == "max":
                mx = float(p[1])
            elif p and p[0] == "error":
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "error": ln[6:]}
            elif len(p) == 3:
                rows.append((float(p[0]), float(p[1]), int(p[2])))
        inside = [r for r in rows if any(a <= r[0] <= b for a, b in self.windows)]
        reasons = sorted({name for _, _, m in inside for bit, name in _REASONS.items() if m & bit})
        sm = [r[1] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(sm), "source": "NVML every ~2 ms, samples inside the timed windows"}


# ---------------------------------------------------------------------------
# multi-GPU plumbing (replicas)
# ---------------------------------------------------------------------------
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


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def measure_form(c, storage, inputs, args, world, clk, barrier):
    """Time one storage form on case `c`: the sequential loop (per-step phase
    and step-kernel events) and the product's run(); returns (record, lat, dem)."""
    import torch
    from lbdem_taichi_b200 import _native as Nat
    sub = c["sub"]
    cells = int(np.prod(c["shape"]))
    lat, dem = cases.build(c, storage, *inputs)
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        lat.step(sub)
    torch.cuda.synchronize()
    lat.check_status()
    dem.check_status()
    # inputs larger than L2 several times over need no flush; otherwise a
    # 256 MB buffer is rewritten between steps (outside the per-step events)
    pop_gb = 2 * 19 * cells * (4 if cases.split_form(storage)[0] == "f32" else 2) / 1e9
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda") if pop_gb <= 0.5 else None
    mk = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ev_step = [(mk(), mk()) for _ in range(args.steps)]
    ev_phase = [(mk(), mk(), mk()) for _ in range(args.steps)]   # before map, after step kernel, after DEM
    t0, t1 = mk(), mk()
    Nat.reset_launch_count()
    barrier()
    torch.cuda.synchronize()
    with clk.window():
        cpu0 = time.perf_counter()
        t0.record(st)
        for k in range(args.steps):
            if flush is not None:
                flush.fill_(float(k))
            lat._kernel_events = ev_step[k]
            ev_phase[k][0].record(st)
            lat.collide()
            lat.stream()
            ev_phase[k][1].record(st)
            dem.run_substeps(sub)
            ev_phase[k][2].record(st)
        t1.record(st)
        cpu_launch_ms = (time.perf_counter() - cpu0) * 1e3 / args.steps
        torch.cuda.synchronize()
    lat._kernel_events = None
    launches = Nat.launch_count()
    barrier()
    # with a flush the step time is the sum of the per-step events (map to end of DEM)
    ms = t0.elapsed_time(t1) if flush is None else sum(a.elapsed_time(b) for a, _, b in ev_phase)
    ms_seq = ms
    pipelined = flush is None and not args.no_pipeline
    if pipelined:
        lat.run(40, sub)          # run()'s automatic choice is measured here, outside the timed region
        pipelined = bool(lat._pipeline_choice)
        torch.cuda.synchronize()
        Nat.reset_launch_count()
        barrier()
        torch.cuda.synchronize()
        with clk.window():
            t0.record(st)
            cpu0 = time.perf_counter()
            lat.run(args.steps, sub)
            t1.record(st)
            cpu_launch_ms = (time.perf_counter() - cpu0) * 1e3 / args.steps
            torch.cuda.synchronize()
        launches = Nat.launch_count()
        barrier()
        ms = t0.elapsed_time(t1)
    ms = max_over_ranks(ms, world)
    ms_seq = max_over_ranks(ms_seq, world)
    kern_ms = max_over_ranks(statistics.mean(a.elapsed_time(b) for a, b in ev_step), world)
    lbm_ms = statistics.mean(a.elapsed_time(b) for a, b, _ in ev_phase)
    dem_ms = statistics.mean(b.elapsed_time(d) for _, b, d in ev_phase)
    lat.check_status()
    dem.check_status()
    peak, peak_kind = peaks()
    bpc = BYTES_PER_CELL[storage]
    achieved = bpc * cells / (kern_ms * 1e-3) / 1e9
    rec = {
        "value": round(job_mlups(world, cells, args.steps, ms), 2), "ms_per_step": round(ms / args.steps, 4),
        "pipelined": pipelined,
        "pipeline_probe_ms": [round(v, 4) for v in lat._pipeline_probe] if lat._pipeline_probe else None,
        "sequential": {"value": round(job_mlups(world, cells, args.steps, ms_seq), 2),
                       "ms_per_step": round(ms_seq / args.steps, 4)},
        "kernel_ms": round(kern_ms, 4),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "kernel": f"lbdem_psc_step_{cases.split_form(storage)[0]}", "kernel_ms": round(kern_ms, 4),
                     "bytes_per_cell": bpc,
                     "traffic": round(TRAFFIC_PER_CELL[storage] * cells / 1e9, 4) if storage in TRAFFIC_PER_CELL
                     else None,
                     "traffic_per_cell": TRAFFIC_PER_CELL.get(storage),
                     "traffic_unit": "GB per launch (ncu DRAM read+write per cell of a 192^3 launch x cells)",
                     "traffic_over_algorithmic": (round(TRAFFIC_PER_CELL[storage] / bpc, 3)
                                                  if storage in TRAFFIC_PER_CELL else None)},
        "phases_ms": {"map+step": round(lbm_ms, 4), "step_kernel": round(kern_ms, 4),
                      f"dem_{sub}_substeps": round(dem_ms, 4), "host_launch_per_step": round(cpu_launch_ms, 4)},
        "gpu_launches": launches,
        "l2": (f"inputs larger than L2 (populations {pop_gb:.2f} GB); no flush" if flush is None else
               f"populations {pop_gb:.2f} GB; L2 flushed between steps (256 MB rewrite outside the step events)"),
    }
    return rec, lat, dem


def end_to_end(c, lat, dem, args, world, clk, barrier):
    """The same loop through the public API with host buffers: every step
    uploads the particle state from pinned host memory, steps, and reads back
    the per-particle fluid force/torque and the new state."""
    import torch
    n = c["n"]
    st = torch.cuda.current_stream()
    h_in = torch.empty((2, n, 3), dtype=torch.float64).pin_memory()
    h_out = torch.empty((4, n, 3), dtype=torch.float64).pin_memory()
    h_in[0].copy_(dem._t["position"])
    h_in[1].copy_(dem._t["velocity"])
    torch.cuda.synchronize()
    e_steps = max(1, args.steps // 2)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clk.window():
        tw0 = time.perf_counter()
        e0.record(st)
        for _ in range(e_steps):
            dem._t["position"].copy_(h_in[0], non_blocking=True)
            dem._t["velocity"].copy_(h_in[1], non_blocking=True)
            dem._touched("position")
            lat.step(c["sub"])
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
    cells = int(np.prod(c["shape"]))
    return {"value": round(job_mlups(world, cells, e_steps, e2e_ms), 2), "unit": "MLUPS",
            "h2d_bytes_per_step": 2 * n * 3 * 8, "d2h_bytes_per_step": 4 * n * 3 * 8, "steps": e_steps}


def record_run(c, storage, inputs, steps, drag_steps=(), state_steps=(), plane_steps=(), plane_axis=2,
               plane_index=0):
    """Run case `c` for `steps` coupled steps in `storage` and record what the
    FP64 records of tests/golden/make_fullsize.py hold: per-step total drag and
    torque, per-particle drag at `drag_steps`, particle state at `state_steps`
    and a velocity plane at `plane_steps`."""
    import torch
    lat, dem = cases.build(c, storage, *inputs)
    n = c["n"]
    ff, mf = dem._t["force_fluid"], dem._t["moment_fluid"]
    tot = torch.empty((steps, 2, 3), dtype=torch.float64, device="cuda")
    per = torch.empty((len(drag_steps), n, 3), dtype=torch.float64, device="cuda")
    st_pos = torch.empty((len(state_steps), n, 3), dtype=torch.float64, device="cuda")
    st_vel = torch.empty_like(st_pos)
    dset, sset = {s: k for k, s in enumerate(drag_steps)}, {s: k for k, s in enumerate(state_steps)}
    planes = []
    for s in range(1, steps + 1):
        lat.collide()
        lat.stream()
        tot[s - 1, 0] = ff.sum(0)
        tot[s - 1, 1] = mf.sum(0)
        if s in dset:
            per[dset[s]] = ff
        if s in plane_steps:
            sl = [slice(None)] * 3
            sl[plane_axis] = plane_index
            planes.append(lat.vel.to_numpy()[tuple(sl)].astype(np.float32))
        dem.run_substeps(c["sub"])
        if s in sset:
            st_pos[sset[s]] = dem._t["position"]
            st_vel[sset[s]] = dem._t["velocity"]
    torch.cuda.synchronize()
    lat.check_status()
    dem.check_status()
    out = {"drag_total": tot[:, 0].cpu().numpy(), "torque_total": tot[:, 1].cpu().numpy(),
           "drag": per.cpu().numpy(), "pos": st_pos.cpu().numpy(), "vel": st_vel.cpu().numpy(),
           "u_plane": np.array(planes)}
    del lat, dem
    torch.cuda.empty_cache()
    return out


def drag_errors(rec, ref):
    """Per-step errors of a recorded run against the FP64 record.

    total_scaled[s] = |sum_i F_i - sum_i F64_i| / sum_i |F64_i|: the error of
        the total particle drag relative to the drag scale (the particles' drag
        magnitudes);
    total[s] = |sum_i F_i - sum_i F64_i| / |sum_i F64_i|: the same error relative
        to the total itself, which in the periodic suspension is about 1 % of the
        drag scale (the particles' drags cancel), so it reports that
        cancellation more than the arithmetic (FP32 reaches 1e-2 by it);
    particle[k] = sum_i |F_i - F64_i| / sum_i |F64_i| at the recorded drag steps;
    plane[k] = ||u - u64|| / ||u64|| over the velocity plane;
    position[k] = max_i |x_i - x64_i| (lattice units)."""
    t64 = ref["drag_total"]
    d_tot = np.linalg.norm(rec["drag_total"] - t64, axis=1)
    scale = ref["drag_abs"] if "drag_abs" in ref else np.linalg.norm(ref["drag"], axis=2).sum(axis=1)
    out = {"total_scaled": d_tot / scale, "total": d_tot / np.linalg.norm(t64, axis=1)}
    d64 = ref["drag"].astype(np.float64)
    out["particle"] = (np.linalg.norm(rec["drag"] - d64, axis=2).sum(axis=1) /
                       np.linalg.norm(d64, axis=2).sum(axis=1))
    if len(ref["u_plane"]) and len(rec["u_plane"]):
        u64 = ref["u_plane"].astype(np.float64)
        out["plane"] = (np.sqrt(((rec["u_plane"] - u64) ** 2).sum(axis=(1, 2, 3))) /
                        np.sqrt((u64 ** 2).sum(axis=(1, 2, 3))))
    if len(ref["pos"]) and len(rec["pos"]):
        out["position"] = np.abs(rec["pos"] - ref["pos"]).max(axis=(1, 2))
    return out


def load_record(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


def drag_summary(c, storage, ref):
    inputs = (ref["pos0"], ref["rad"], ref["vel0"], ref["mass"])
    rec = record_run(c, storage, inputs, int(ref["steps"]), list(ref["drag_steps"]), list(ref["state_steps"]),
                     list(ref["plane_steps"]), int(ref["plane_axis"]), int(ref["plane_index"]))
    e = drag_errors(rec, ref)
    sc, lit = e["total_scaled"], e["total"]
    return {"drag_rel_err_vs_fp64": float(sc.max()), "worst_step": int(np.argmax(sc)) + 1,
            "drag_rel_err_definition": "max over steps of |sum F - sum F64| / sum |F64| (total drag error relative "
                                       "to the particles' drag magnitudes)",
            "steps_within_1e-3": f"{int((sc <= 1e-3).sum())}/{len(sc)}",
            "total_drag_rel_err_vs_total": {"max": float(lit.max()), "median": float(np.median(lit)),
                                            "first_step_above_1e-3": (int(np.argmax(lit > 1e-3)) + 1
                                                                      if (lit > 1e-3).any() else None)},
            "particle_drag_rel_err_max": float(e["particle"].max()),
            "velocity_plane_rel_err": [float(v) for v in e.get("plane", [])],
            "position_err_max_lu": float(e["position"].max()) if "position" in e else None,
            "steps": int(ref["steps"]),
            "reference": "FP64 oracle record of the same run (tests/golden/c2_fp64.npz)"}


def run_gpu(c, args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    clk = Clocks(local)

    def barrier():
        if world > 1:
            dist.barrier()

    inputs = cases.particles(c)
    clk.wait_ready()
    head, lat, dem = measure_form(c, args.storage, inputs, args, world, clk, barrier)
    e2e = end_to_end(c, lat, dem, args, world, clk, barrier)
    del lat, dem
    torch.cuda.empty_cache()
    forms = {args.storage: head}
    if not args.no_forms:
        for storage in FORMS:
            if storage not in forms:
                forms[storage], lat, dem = measure_form(c, storage, inputs, args, world, clk, barrier)
                del lat, dem
                torch.cuda.empty_cache()
    full_c2 = c["key"] == "c2" and c["shape"] == cases.CASES["c2"]["shape"] and c["n"] == cases.CASES["c2"]["n"]
    ref = load_record(FIXTURE) if (full_c2 and not args.no_drag and os.path.exists(FIXTURE)) else None
    storage_forms = {}
    base = forms.get("f32")
    for storage, r in forms.items():
        f = {"value": r["value"], "unit": "MLUPS", "ms_per_step": r["ms_per_step"], "kernel_ms": r["kernel_ms"],
             "roofline_frac": r["roofline"]["frac"], "achieved_gbs": r["roofline"]["achieved"],
             "traffic_per_cell": r["roofline"]["traffic_per_cell"], "pipelined": r["pipelined"]}
        if base is not None:
            f["kernel_speedup_vs_f32"] = round(base["kernel_ms"] / r["kernel_ms"], 3)
            f["step_speedup_vs_f32"] = round(base["ms_per_step"] / r["ms_per_step"], 3)
        if ref is not None:
            f.update(drag_summary(c, storage, ref))
        storage_forms[storage] = f
    cells = int(np.prod(c["shape"]))
    out = {
        "metric": METRIC, "value": head["value"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": {"workload": c["desc"], "name": c["key"], "lattice": list(c["shape"]), "cells": cells,
                   "particles": c["n"], "dem_subcycles": c["sub"], "storage": args.storage, "l2": head["l2"],
                   "parallelism": f"replicas x{world}"},
        "roofline": head["roofline"],
        "e2e": e2e,
        "gpu_launches": head["gpu_launches"],
        "pipelined": head["pipelined"],
        "pipeline_probe_ms": head["pipeline_probe_ms"],
        "sequential": head["sequential"],
        "phases_ms": head["phases_ms"],
        "storage_forms": storage_forms,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(c, inputs, budget_s=args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# CPU arm: the FP64 C restatement of the reference path (oracle/), timed on
# the host cores.  The reference's grains2lattice probes every particle for
# every cell, so a full-size step is sampled: the lattice part (map with the
# reference's all-grains loop, collision, force reduction, streaming) on a
# z-slab of the lattice that carries every particle gives the time per cell,
# and the DEM part (10 sub-steps of all particles) the time per step; the two
# recombine into the full lattice's step time.
# ---------------------------------------------------------------------------
SLAB_Z = 4


def cpu_sample(c, inputs, nz_slab):
    from oracle.oracle import OracleDEM, OracleGrains, OracleLattice
    nx, ny, nz = c["shape"]
    pos, rad, vel, mass = inputs
    lat = OracleLattice(nx, ny, nz_slab, 1.0 / c["tau"], smag=c["cs"] is not None, psc=True,
                        force=c["fluid_force"], smag_cs=c["cs"] if c["cs"] is not None else 0.1)
    lat.ct[...] = cases.cell_types(c)[:, :, :nz_slab]
    if "u_in" in c:
        cases.open_presets(c, lat.vel, lat.rho)
    h, e = cases.HERTZ, cases.ELASTIC
    dem = OracleDEM(pos, vel, rad, mass, dt=1.0 / c["sub"], gravity=c["gravity"], domain=(0, nx, 0, ny, 0, nz),
                    periodic=("u_in" not in c, True, not c["walls_z"]), E=e["E"], nu=e["nu"], wall_E=e["E"],
                    wall_nu=e["nu"], pp_mu=h["pp_friction"], pw_mu=h["pw_friction"], pp_e=h["pp_restitution"],
                    pw_e=h["pw_restitution"], max_coord=cases.MAX_COORD)
    g = OracleGrains(dem.pos, dem.radius, dem.vel, dem.omega)
    g.force_fluid, g.moment_fluid = dem.force_fluid, dem.moment_fluid
    lat.initialize()
    return lat, dem, g


def cpu_step(c, lat, dem, g):
    """(lattice seconds, DEM seconds) of one sampled step."""
    t0 = time.perf_counter()
    lat.grains2lattice_all(g)
    lat.collide()
    lat.lattice2grains(g)
    lat.stream()
    t1 = time.perf_counter()
    for _ in range(c["sub"]):
        dem.run_simulation()
    return t1 - t0, time.perf_counter() - t1


def _full_mlups(c, nz_slab, lat_s, dem_s):
    """MLUPS of a full-lattice step from a slab's lattice time and a DEM time."""
    nx, ny, nz = c["shape"]
    cells = nx * ny * nz
    step_s = lat_s / (nx * ny * nz_slab) * cells + dem_s
    return cells / step_s / 1e6, step_s


def _sample_text(c, nz_slab, steps):
    nx, ny, _ = c["shape"]
    return (f"{steps} sampled steps: lattice part (reference all-grains map, collide, force reduction, stream) on a "
            f"{nx}x{ny}x{nz_slab} slab carrying all {c['n']} particles, timed per cell; DEM part ({c['sub']} "
            f"sub-steps of all particles) timed per step; recombined for the full {c['shape'][0]}x{c['shape'][1]}x"
            f"{c['shape'][2]} lattice; FP64 C restatement, OpenMP {os.cpu_count()} threads")


def cpu_baseline(c, inputs, budget_s=20.0):
    nz_slab = min(SLAB_Z, c["shape"][2])
    lat, dem, g = cpu_sample(c, inputs, nz_slab)
    cpu_step(c, lat, dem, g)     # first touch of the oracle's arrays
    t0 = time.perf_counter()
    lat_s, dem_s, steps = 0.0, 0.0, 0
    while time.perf_counter() - t0 < budget_s * 0.5 and steps < 50:
        a, b = cpu_step(c, lat, dem, g)
        lat_s, dem_s, steps = lat_s + a, dem_s + b, steps + 1
    v, step_s = _full_mlups(c, nz_slab, lat_s / steps, dem_s / steps)
    return {"value": round(v, 4), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
            "ms_per_full_step": round(step_s * 1e3, 1), "sample": _sample_text(c, nz_slab, steps)}


def run_reference(c, args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    inputs = cases.particles(c)
    nz_slab = min(SLAB_Z, c["shape"][2])
    lat, dem, g = cpu_sample(c, inputs, nz_slab)
    for _ in range(args.warmup):
        cpu_step(c, lat, dem, g)
    lat_s = dem_s = 0.0
    for _ in range(args.steps):
        a, b = cpu_step(c, lat, dem, g)
        lat_s, dem_s = lat_s + a, dem_s + b
    steps = max(1, args.steps)
    v, step_s = _full_mlups(c, nz_slab, lat_s / steps, dem_s / steps)
    sample = _sample_text(c, nz_slab, args.steps)
    nx, ny, nz = c["shape"]
    # the GPU arm's config; the reference computes in FP64 on the host cores (no GPU)
    out = {"metric": METRIC, "value": round(v, 4), "unit": "MLUPS", "impl": "reference", "n_gpus": args.gpus,
           "device": "cpu", "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(step_s * 1e3, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": c["desc"], "name": c["key"], "lattice": [nx, ny, nz], "cells": nx * ny * nz,
                      "particles": c["n"], "dem_subcycles": c["sub"], "storage": "f64",
                      "sample": f"per step: {sample}", "parallelism": f"{os.cpu_count()} host threads"},
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
ADJ_N, ADJ_NP, ADJ_STEPS, ADJ_EVERY, ADJ_G, ADJ_TAU = 128, 500, 500, 50, 2e-6, 0.6


def adjoint_workload(seed=2024):
    rng = np.random.default_rng(seed)
    pos, rad = cases.rsa_spheres(rng, ADJ_NP, (ADJ_N, ADJ_N, ADJ_N), 10.0, 10.0, gap=0.2, zmax=ADJ_N / 2,
                                 margin=1.0)
    ct = np.full((ADJ_N,) * 3, 1, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = 8
    return pos, rad, ct


def run_adjoint(args):
    import torch

    from lbdem_taichi_b200 import _native as Nat
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from lbdem_taichi_b200.lbdem.adjoint import FrozenBedDrag
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    pos, rad, ct = adjoint_workload()
    n = len(rad)
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    dem = cases.make_dem((0.0, ADJ_N, 0.0, ADJ_N, 0.0, ADJ_N), 0.1, (0, 0, 0), HertzContactConfig(**cases.HERTZ),
                         rad, mass, pos, np.zeros((n, 3)), periodic=(True, True, False),
                         freeze=np.ones(n, np.int32))
    lat = PSCLattice3D(ADJ_N, ADJ_N, ADJ_N, 1.0 / ADJ_TAU, 1.0, 1.0, 1.0, dem, body_force=(ADJ_G, 0.0, 0.0),
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
            return frozen_bed_drag(shape, 1.0 / ADJ_TAU, ct, rad, P, Fv, ADJ_STEPS)
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
    ap.add_argument("--storage", default="f32", choices=list(FORMS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pipeline", action="store_true", help="time the sequential loop (collide, stream, DEM)")
    ap.add_argument("--no-forms", action="store_true", help="time only --storage, not every storage form")
    ap.add_argument("--no-drag", action="store_true", help="skip the drag error against the FP64 record")
    ap.add_argument("--workload", default="c2", choices=sorted(cases.CASES))
    ap.add_argument("--size", type=int, default=0, help="cube edge override; only for small profiling cases")
    ap.add_argument("--particles", type=int, default=0, help="particle count override; only for profiling")
    ap.add_argument("--adjoint", action="store_true", help="drag-gradient workload instead of the step")
    ap.add_argument("--adjoint-fd", type=int, default=0, help="FP64 finite-difference checks (count)")
    args = ap.parse_args()
    if args.adjoint:
        run_adjoint(args)
        return
    c = cases.case(args.workload, args.size, args.particles)
    if args.impl == "reference":
        run_reference(c, args)
    else:
        run_gpu(c, args)


if __name__ == "__main__":
    main()
