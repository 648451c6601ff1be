"""FP64 records of the full-size cases, written by the oracle.

    python tests/golden/make_fullsize.py [c2] [c1] [--steps N]

c2 (``c2_fp64.npz``): the dense suspension at its full size -- 256^3, periodic,
2000 spheres d ~ U[8, 12], Hertz, body force 1e-6, tau 0.6, Smagorinsky 0.1
in the reference's lagged form, 10 DEM sub-steps -- over 1000 coupled steps.
c1 (``c1_fp64.npz``): one sphere d = 12 settling in 64 x 64 x 128 between
walls, 2000 steps.  Both start from the seeded inputs of
``lbdem_taichi_b200.cases`` (the same ones the GPU tests and bench.py build).

The oracle is the FP64 C restatement of the reference path in ``oracle/``
(pinned to golden vectors of the reference's own source).  Its map visits each
cell's grains through 8^3-cell bins, which gives exactly the reference's
per-cell loop over all grains (``tests/test_oracle_map_bins.py``) at a cost
that does not grow with cells x grains, so these sizes run in minutes.

A step is the reference driver loop (single_particle_settle.py:235-240):
grains2lattice, collide, lattice2grains, stream, then the DEM sub-steps.
Records per step ``s`` (1-based; the drag is the one the step's collision
gives, i.e. the force the following DEM sub-steps use):
  drag_total[s-1]    sum over particles of force_fluid (3)
  torque_total[s-1]  sum over particles of moment_fluid (3)
  drag_abs[s-1]      sum over particles of |force_fluid|
  sums[s-1]          FP64 mass and momentum of the fluid after streaming
  drag[k]            per-particle force_fluid at drag_steps[k] (float32)
  pos[k], vel[k]     particle state after the DEM sub-steps at state_steps[k]
  u_plane[k]         fluid velocity of the plane ``plane_axis = plane_index``
                     after streaming at plane_steps[k] (float32)
c1 additionally keeps the particle's position, velocity, force and torque of
every step.  Runtime on 8 host cores: about 15 minutes for c2, 1 for c1.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lbdem_taichi_b200 import cases  # noqa: E402
from oracle.oracle import OracleDEM, OracleGrains, OracleLattice  # noqa: E402

SEED = 2024
SPEC = {
    "c2": dict(steps=1000, drag_steps=list(range(1, 10)) + list(range(10, 1001, 10)),
               state_steps=list(range(100, 1001, 100)), plane_steps=[100, 500, 1000], plane_axis=2,
               plane_index=128),
    "c1": dict(steps=2000, drag_steps=list(range(1, 2001)), state_steps=list(range(1, 2001)),
               plane_steps=[500, 1000, 2000], plane_axis=1, plane_index=32),
}


def oracle_case(c, pos, rad, vel, mass):
    """Oracle lattice, DEM and grain view of case `c` (the parameters of
    ``cases.build``, in the oracle's terms)."""
    nx, ny, nz = c["shape"]
    lat = OracleLattice(nx, ny, nz, 1.0 / c["tau"], smag=c["cs"] is not None, psc=True, force=c["fluid_force"],
                        smag_cs=c["cs"] if c["cs"] is not None else 0.1)
    lat.ct[...] = cases.cell_types(c)
    h, e = cases.HERTZ, cases.ELASTIC
    dem = OracleDEM(pos, vel, rad, mass, dt=1.0 / c["sub"], gravity=c["gravity"], domain=(0, nx, 0, ny, 0, nz),
                    periodic=(True, True, not c["walls_z"]), E=e["E"], nu=e["nu"], wall_E=e["E"], wall_nu=e["nu"],
                    pp_mu=h["pp_friction"], pw_mu=h["pw_friction"], pp_e=h["pp_restitution"],
                    pw_e=h["pw_restitution"], max_coord=cases.MAX_COORD)
    g = OracleGrains(dem.pos, dem.radius, dem.vel, dem.omega)
    g.force_fluid, g.moment_fluid = dem.force_fluid, dem.moment_fluid
    lat.initialize()
    return lat, dem, g


def record(name, steps=None):
    spec = dict(SPEC[name])
    if steps:
        spec["steps"] = steps
    n_steps = spec["steps"]
    c = cases.case(name)
    pos, rad, vel, mass = cases.particles(c, SEED)
    lat, dem, g = oracle_case(c, pos, rad, vel, mass)
    drag_steps = [s for s in spec["drag_steps"] if s <= n_steps]
    state_steps = [s for s in spec["state_steps"] if s <= n_steps]
    plane_steps = [s for s in spec["plane_steps"] if s <= n_steps]
    out = {k: [] for k in ("drag_total", "torque_total", "drag_abs", "sums", "drag", "pos", "vel", "u_plane")}
    t0 = time.time()
    for s in range(1, n_steps + 1):
        lat.grains2lattice(g)
        lat.collide()
        lat.lattice2grains(g)
        lat.stream()
        out["drag_total"].append(dem.force_fluid.sum(axis=0))
        out["torque_total"].append(dem.moment_fluid.sum(axis=0))
        out["drag_abs"].append(np.linalg.norm(dem.force_fluid, axis=1).sum())
        out["sums"].append(lat.global_sums())
        if s in drag_steps:
            out["drag"].append(dem.force_fluid.astype(np.float32))
        if s in plane_steps:
            sl = [slice(None)] * 3
            sl[spec["plane_axis"]] = spec["plane_index"]
            out["u_plane"].append(lat.vel[tuple(sl)].astype(np.float32))
        for _ in range(c["sub"]):
            dem.run_simulation()
        assert dem.status == 0, f"oracle DEM status {dem.status} at step {s}"
        if s in state_steps:
            out["pos"].append(dem.pos.copy())
            out["vel"].append(dem.vel.copy())
        if s % 50 == 0:
            print(f"{name}: step {s}/{n_steps}  {time.time() - t0:.0f} s  |F| {out['drag_abs'][-1]:.4e}",
                  flush=True)
    rec = {k: np.asarray(v) for k, v in out.items()}
    rec.update(seed=SEED, steps=n_steps, drag_steps=np.asarray(drag_steps), state_steps=np.asarray(state_steps),
               plane_steps=np.asarray(plane_steps), plane_axis=spec["plane_axis"],
               plane_index=spec["plane_index"], pos0=pos, rad=rad, vel0=vel, mass=mass)
    path = os.path.join(HERE, f"{name}_fp64.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.1f} MB) in {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    steps = int(sys.argv[sys.argv.index("--steps") + 1]) if "--steps" in sys.argv else None
    args = [a for a in args if not a.isdigit()]
    for name in args or ["c1", "c2"]:
        record(name, steps)
