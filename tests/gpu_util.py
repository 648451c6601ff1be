"""Builders shared by the GPU tests: the same scenarios as the golden
fixtures / oracle, constructed through the product's Python API."""
import numpy as np

from lbdem_taichi_b200 import Vector3
from lbdem_taichi_b200.dem3d.demconfig import (DEMSolverConfig, DomainBounds, HertzContactConfig,
                                               LinearContactConfig)
from lbdem_taichi_b200.dem3d.demsolver import DEMSolver


def make_dem(domain, dt, gravity, contact, radius, mass, pos, vel, omega=None, periodic=(False, False, False),
             E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3, max_coord=16, model="hertz", freeze=None, compat="reference"):
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


def golden_dem(g, model):
    contact = (HertzContactConfig(pp_friction=0.3, pw_friction=0.4, pp_restitution=0.9, pw_restitution=0.8)
               if model == "hertz" else
               LinearContactConfig(stiffness_normal=200.0, stiffness_tangential=100.0, damping_normal=0.2,
                                   damping_tangential=0.1, pp_friction=0.3, pw_friction=0.4))
    return make_dem(g["domain"], float(g["dt"]), g["gravity"], contact, g["grad"], g["mass"], g["gpos"], g["gvel"],
                    omega=g["gomega"], periodic=tuple(bool(v) for v in g["periodic"]), E=float(g["E"]),
                    nu=float(g["nu"]), wall_E=float(g["wall_E"]), wall_nu=float(g["wall_nu"]),
                    max_coord=int(g["max_coord"]), model=model)


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
