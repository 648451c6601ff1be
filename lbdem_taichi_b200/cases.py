"""Seeded synthetic versions of the reference's LBM-DEM driver set-ups.

The reference's example drivers (``example/lbdem/single_particle_settle``,
``shear_suspensions``, ``pressure_dropfully_1``) build a lattice, read or place
particles and loop ``collide(); stream(); dem.run_simulation()``.  The cases
here are the same kind of set-up with seeded random inputs instead of the
drivers' literature particle files (none of which is shipped), built through
the public API (``PSCLattice3D``, ``DEMSolver``).  All values are in lattice
units (dx = dt = rho0 = 1).

    c2     dense suspension: 256^3 periodic, 2000 spheres d ~ U[8, 12] placed by
           random sequential addition with a 1 lu gap, Gaussian velocities
           (sigma 1e-3), density ratio 2.0, Hertz e = 0.9, body force 1e-6 (x)
           on fluid and particles, tau 0.6, Smagorinsky Cs 0.1 (lagged form)
    c5     512 x 512 x 256 channel, walls at z = 0 and 255, 20000 spheres
           d ~ U[6, 10], tau 0.51, Cs 0.12
    c1     one sphere d = 12 settling in 64 x 64 x 128 between walls at
           z = 0 and 127, density ratio 2.5, gravity 1e-5 (buoyancy-reduced)
    pdrop  packed-bed pressure drop, 722 x 242 x 242: Ladd velocity inlet,
           Zou-He pressure outlet, 1500 frozen spheres d = 24, linear contacts

Parameters the set-ups leave open (friction 0.3, E = 1e5, nu = 0.3,
10 DEM sub-steps per lattice step, 16 contact slots per particle) are fixed
here and used identically by every consumer.
"""
from __future__ import annotations

import numpy as np

CASES = {
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

# Contact parameters of every case (linear: the packed bed's driver values)
HERTZ = dict(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)
LINEAR = dict(stiffness_normal=4.5e3, stiffness_tangential=2.5e3, damping_normal=0.3, damping_tangential=0.2,
              pp_friction=0.15, pw_friction=0.15)
ELASTIC = dict(E=1e5, nu=0.3)
MAX_COORD = 16


def case(name: str, size: int = 0, particles: int = 0) -> dict:
    """The case's parameters; `size` (cube edge) and `particles` shrink it for
    profiling on small lattices."""
    c = dict(CASES[name], key=name)
    if size:
        c["shape"] = (size, size, size)
    if particles:
        c["n"] = particles
    return c


def rsa_spheres(rng, n, box, dmin_, dmax_, gap=1.0, zmax=None, margin=0.0, tries=200000):
    """Seeded random sequential addition of non-overlapping spheres in a box
    (lattice units); returns centres and radii."""
    pos, rad = [], []
    lo = np.array([margin, margin, margin], float)
    hi = np.array(box, float) - margin
    if zmax is not None:
        hi[2] = min(hi[2], zmax)
    for _ in range(tries):
        if len(rad) == n:
            break
        r = 0.5 * rng.uniform(dmin_, dmax_)
        p = rng.uniform(lo + r, hi - r)
        if rad:
            P = np.array(pos)
            R = np.array(rad)
            if np.any(np.linalg.norm(P - p, axis=1) < R + r + gap):
                continue
        pos.append(p)
        rad.append(r)
    if len(rad) < n:
        raise RuntimeError(f"RSA placed only {len(rad)} of {n} spheres")
    return np.array(pos), np.array(rad)


def rsa_spheres_grid(rng, n, box, dmin_, dmax_, gap=1.0, zmin=None, zmax=None, margin=0.0, tries=5000000):
    """rsa_spheres for large counts: the same seeded sequential addition with a
    hash grid of cell size (dmax + gap) for the overlap test."""
    lo = np.array([margin, margin, margin], float)
    hi = np.array(box, float) - margin
    if zmin is not None:
        lo[2] = max(lo[2], zmin)
    if zmax is not None:
        hi[2] = min(hi[2], zmax)
    cs = dmax_ + gap
    grid = {}
    pos, rad = [], []
    for _ in range(tries):
        if len(rad) == n:
            break
        r = 0.5 * rng.uniform(dmin_, dmax_)
        p = rng.uniform(lo + r, hi - r)
        c = np.floor(p / cs).astype(int)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        if np.sum((pos[j] - p) ** 2) < (rad[j] + r + gap) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault((c[0], c[1], c[2]), []).append(len(rad))
        pos.append(p)
        rad.append(r)
    if len(rad) < n:
        raise RuntimeError(f"RSA placed only {len(rad)} of {n} spheres")
    return np.array(pos), np.array(rad)


def particles(c: dict, seed: int = 2024):
    """Seeded particle centres, radii, velocities and masses of case `c`."""
    nx, ny, nz = c["shape"]
    n = c["n"]
    rng = np.random.default_rng(seed)
    if c["key"] == "c1":
        pos = np.array([[nx / 2 + rng.uniform(-0.5, 0.5), ny / 2 + rng.uniform(-0.5, 0.5), nz - 18.0]])
        rad = np.array([0.5 * c["dmin"]])
    elif "u_in" in c:
        xc = c["x_clear"]
        pos, rad = rsa_spheres_grid(rng, n, (nx - 2 * xc, ny, nz), c["dmin"], c["dmax"], gap=c["gap"], margin=0.5)
        pos[:, 0] += xc
    else:
        zlo = 1.0 if c["walls_z"] else None
        zhi = nz - 1.0 if c["walls_z"] else None
        pos, rad = rsa_spheres_grid(rng, n, (nx, ny, nz), c["dmin"], c["dmax"], gap=c["gap"], zmin=zlo, zmax=zhi,
                                    margin=0.5)
    vel = rng.normal(0.0, c["vel_sigma"], (n, 3)) if c["vel_sigma"] > 0 else np.zeros((n, 3))
    mass = c["rho_p"] * 4.0 / 3.0 * np.pi * rad ** 3
    return pos, rad, vel, mass


def cell_types(c: dict):
    """CellType field (Nx, Ny, Nz) of case `c`: FLUID, OBSTACLE walls, open faces."""
    nx, ny, nz = c["shape"]
    ct = np.full((nx, ny, nz), 1, np.int32)
    if c["walls_z"]:
        ct[:, :, 0] = ct[:, :, -1] = 8
    if "u_in" in c:
        ct[0] = 262144 | 8192     # VEL_INLET_LADD | LEFT
        ct[-1] = 256 | 4096       # Pre_ZOUHE | RIGHT
    return ct


def open_presets(c: dict, vel, rho):
    """Inlet velocity and outlet density of an open-boundary case (in place)."""
    vel[0, ..., 0] = c["u_in"]
    rho[-1] = 1.0


def make_dem(domain, dt, gravity, contact, radius, mass, pos, vel, omega=None, periodic=(False, False, False),
             E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3, max_coord=16, model="hertz", freeze=None, compat="reference"):
    """DEMSolver over the given particle arrays (the reference's
    DEMSolverConfig / set_* / init_particle_fields sequence)."""
    from . import Vector3
    from .dem3d.demconfig import DEMSolverConfig, DomainBounds
    from .dem3d.demsolver import DEMSolver
    cfg = DEMSolverConfig(domain=DomainBounds(*[float(v) for v in domain]), dt=dt, gravity=Vector3(*gravity),
                          contact_model=contact)
    cfg.set_particle_properties(elastic_modulus=E, poisson_ratio=nu, max_coordinate_number=max_coord)
    cfg.set_wall_properties(elastic_modulus=wall_E, poisson_ratio=wall_nu)
    cfg.set_periodic_boundaries(*periodic)
    dem = DEMSolver(cfg, compat=compat)
    dmin = Vector3(domain[0], domain[2], domain[4])
    dmax = Vector3(domain[1], domain[3], domain[5])
    dem.init_particle_arrays(radius, mass, pos, vel, dmin, dmax)
    if omega is not None:
        dem.gf.omega.from_numpy(np.asarray(omega))
    if freeze is not None:
        dem.gf.freeze.from_numpy(np.asarray(freeze, np.int32))
    dem.set_contact_model(model)
    return dem


def split_form(form: str):
    """(storage, lagged_storage) of a storage-form name: "f32", "f16", "bf16",
    or "f32-lag16" (FP32 populations, FP16 lagged Smagorinsky state)."""
    if form == "f32-lag16":
        return "f32", "f16"
    return form, None


def build(c: dict, storage: str, pos, rad, vel, mass):
    """(PSCLattice3D, DEMSolver) of case `c`, initialised, in storage form
    `storage` (``split_form``)."""
    storage, lagged = split_form(storage)
    from .dem3d.demconfig import HertzContactConfig, LinearContactConfig
    from .lbdem.psclattice3d import PSCLattice3D
    nx, ny, nz = c["shape"]
    opened = "u_in" in c
    contact = LinearContactConfig(**LINEAR) if opened else HertzContactConfig(**HERTZ)
    dem = make_dem((0.0, float(nx), 0.0, float(ny), 0.0, float(nz)), 1.0 / c["sub"], c["gravity"], contact, rad,
                   mass, pos, vel, periodic=(not opened, True, not c["walls_z"]), E=ELASTIC["E"], nu=ELASTIC["nu"],
                   wall_E=ELASTIC["E"], wall_nu=ELASTIC["nu"], max_coord=MAX_COORD,
                   model="linear" if opened else "hertz",
                   freeze=np.ones(len(rad), np.int32) if opened else None)
    lat = PSCLattice3D(nx, ny, nz, 1.0 / c["tau"], 1.0, 1.0, 1.0, dem,
                       smagorinsky="off" if c["cs"] is None else "reference", body_force=c["fluid_force"],
                       storage=storage, lagged_storage=lagged)
    if c["cs"] is not None:
        lat.SmagorinskyConstant = c["cs"]
    if c["walls_z"] or opened:
        lat.CT.from_numpy(cell_types(c))
    if opened:
        v, r = lat.vel.to_numpy(), lat.rho.to_numpy()
        open_presets(c, v, r)
        lat.vel.from_numpy(v)
        lat.rho.from_numpy(r)
    lat.initialize()
    return lat, dem
