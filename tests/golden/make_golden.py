"""Generate golden fixtures by running the reference's OWN Python source
(dasfadwqd/LBDEM-Taichi, from a checkout given on the command line) under the NumPy Taichi
stand-in in ``tishim.py``.

Usage (in a container that has the reference checkout):
    python tests/golden/make_golden.py <reference checkout>     (or LBDEM_REFERENCE=<checkout>)

Every scenario writes ``tests/golden/<name>.npz``.  Inputs are seeded; all
arrays keep the reference's own shapes ((Nx, Ny, Nz[, k]) for lattice fields,
(n, ...) for particle fields).

Two reference routines are replaced by vectorised equivalents because a
Python-loop emulation of them over the reference's 2^20-entry hash table
would take minutes per DEM sub-step; both replacements compute identical
integers:
  * ``BPCD._setup_collision`` (bpcd.py:105-112): clear the table, then count
    particles per hash cell -- the count loop still calls the reference's own
    ``hash_codef``;
  * ``PrefixSumExecutor.parallel_fast`` (prefixsum.py:62-84): exclusive scan.
Everything else (mapping, collision, streaming, force reduction, contact
search, contact laws, walls, integration) is the reference's code as written.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import tishim  # noqa: E402

ti = tishim.install()

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LBDEM_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "src")):
    sys.exit(f"usage: python {os.path.relpath(__file__)} <reference checkout> (or set LBDEM_REFERENCE); "
             "the checkout must hold the reference's src/ package")
sys.path.insert(0, REF)

from src.lbm3d.lbm_solver3d import BasicLattice3D  # noqa: E402
from src.lbm3d.lbm_foecelover import ForcedLattice3D  # noqa: E402
from src.lbm3d.lbmutils import CellType  # noqa: E402
from src.lbdem.psclattice3d import PSCLattice3D  # noqa: E402
from src.hybridlbdem.hybridlattice import HybridLattice3D  # noqa: E402
from src.dem3d.demsolver import DEMSolver  # noqa: E402
from src.dem3d.demconfig import (DEMSolverConfig, DomainBounds,  # noqa: E402
                                 HertzContactConfig, LinearContactConfig)
from src.dem3d.bpcd import BPCD, PrefixSumExecutor  # noqa: E402

Vector3 = ti.types.vector(3, float)


# ---------------------------------------------------------------------------
# vectorised stand-ins for the two table-sized loops (identical integers)
# ---------------------------------------------------------------------------
def _setup_collision_fast(self, positions):
    ht = self.hash_table
    ht.offset.arr[...] = 0
    ht.current.arr[...] = 0
    ht.count.arr[...] = 0
    for i in positions:
        self._count_particles(positions[i])


def _parallel_fast(self, output, input, cal_total=False):
    a = input.arr.astype(np.int64)
    ex = np.concatenate([[0], np.cumsum(a)[:-1]])
    output.arr[...] = ex
    if cal_total:
        return int(ex[-1] + a[-1])


BPCD._setup_collision = _setup_collision_fast
PrefixSumExecutor.parallel_fast = _parallel_fast


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def write_p4p(path, radius, mass, pos, vel):
    """Reference p4p format: single spaces, 1-based IDs (demsolver.py:160-177)."""
    n = len(radius)
    with open(path, "w") as fp:
        fp.write("TIMESTEP  PARTICLES\n")
        fp.write(f"0 {n}\n")
        fp.write("ID  GROUP  RAD  MASS  PX  PY  PZ  VX  VY  VZ\n")
        for i in range(n):
            fp.write(" ".join([str(i + 1), "0", repr(float(radius[i])), repr(float(mass[i])),
                               repr(float(pos[i, 0])), repr(float(pos[i, 1])), repr(float(pos[i, 2])),
                               repr(float(vel[i, 0])), repr(float(vel[i, 1])), repr(float(vel[i, 2]))])
                     + "\n")


def make_dem(domain, dt, gravity, contact, radius, density, pos, vel, omega=None,
             periodic=(False, False, False), E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3,
             max_coord=16, model="hertz", freeze=None):
    mass = density * 4.0 / 3.0 * np.pi * radius ** 3
    cfg = DEMSolverConfig(domain=DomainBounds(*domain), dt=dt, gravity=Vector3(*gravity),
                          contact_model=contact)
    cfg.set_particle_properties(elastic_modulus=E, poisson_ratio=nu, max_coordinate_number=max_coord)
    cfg.set_wall_properties(elastic_modulus=wall_E, poisson_ratio=wall_nu, density=density)
    cfg.set_periodic_boundaries(*periodic)
    fd, path = tempfile.mkstemp(suffix=".p4p")
    os.close(fd)
    write_p4p(path, radius, mass, pos, vel)
    dem = DEMSolver(cfg)
    dmin = Vector3(domain[0], domain[2], domain[4])
    dmax = Vector3(domain[1], domain[3], domain[5])
    dem.init_particle_fields(path, dmin, dmax)
    os.remove(path)
    dem.set_contact_model(model)
    if omega is not None:
        dem.gf.omega.from_numpy(omega)
    if freeze is not None:
        dem.gf.freeze.from_numpy(np.asarray(freeze, dtype=np.int64))
    return dem


def set_walls_z(lattice):
    ct = lattice.CT.arr
    ct[:, :, 0] = CellType.OBSTACLE
    ct[:, :, -1] = CellType.OBSTACLE


def random_flow(lattice, rng, amp_u, amp_rho):
    nx, ny, nz = lattice.Nx, lattice.Ny, lattice.Nz
    lattice.vel.arr[...] = amp_u * rng.uniform(-1, 1, (nx, ny, nz, 3))
    lattice.rho.arr[...] = 1.0 + amp_rho * rng.uniform(-1, 1, (nx, ny, nz))


def dem_state(dem):
    gf = dem.gf
    return {k: getattr(gf, k).to_numpy() for k in (
        "position", "velocity", "acceleration", "force", "quaternion", "omega",
        "omega_dot", "moment", "force_fluid", "moment_fluid")}


def dem_contacts(dem):
    cf = dem.cf
    act = cf.isActive.to_numpy().astype(bool)
    pairs = np.stack([cf.i.to_numpy()[act], cf.j.to_numpy()[act]], 1) if act.any() else np.zeros((0, 2), int)
    shear = cf.shear_displacement.to_numpy()[act]
    wact = dem.wcf.isActive.to_numpy().astype(bool)
    wshear = dem.wcf.shear_displacement.to_numpy()
    return pairs, shear, wact, wshear


def save(name, **arrs):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrs)
    print(f"wrote {path}: {sorted(arrs)}")


# ---------------------------------------------------------------------------
# scenarios
# ---------------------------------------------------------------------------
def scen_bgk_smag():
    """BasicLattice3D.collide (Smagorinsky, lbm_solver3d.py:176-192) + stream."""
    rng = np.random.default_rng(11)
    nx, ny, nz = 10, 8, 7
    lat = BasicLattice3D(nx, ny, nz, 1.0 / 0.6, 1.0, 1.0, 1.0)
    set_walls_z(lat)
    random_flow(lat, rng, 0.05, 0.01)
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy())
    lat.initialize()
    out = {}
    for s in range(3):
        lat.collide()
        out[f"omega_{s}"] = lat.omega.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("bgk_smag", omega0=np.float64(1.0 / 0.6), cs=np.float64(BasicLattice3D.SmagorinskyConstant),
         nsteps=np.int64(3), **init, **out)


def scen_forced():
    """ForcedLattice3D.collide (lbm_foecelover.py:52-68) + stream."""
    rng = np.random.default_rng(12)
    nx, ny, nz = 9, 8, 8
    F = (1e-3, -2e-3, 5e-4)
    lat = ForcedLattice3D(nx, ny, nz, 1.0 / 0.7, 1.0, 1.0, 1.0, Vector3(*F))
    set_walls_z(lat)
    random_flow(lat, rng, 0.02, 0.005)
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy())
    lat.initialize()
    out = {}
    for s in range(3):
        lat.collide()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("forced", omega0=np.float64(1.0 / 0.7), force=np.array(F), nsteps=np.int64(3), **init, **out)


def _psc_particles(dx, xmin):
    # lattice-unit centres (xc as defined at psclattice3d.py:102-104) -> physical
    xc = np.array([[5.3, 5.1, 4.7],     # G0: large, has fully covered cells
                   [9.4, 6.2, 5.5],     # G1: partial overlap with G0 -> winner rule
                   [10.0, 3.0, 2.2],    # G2: near the z=0 wall
                   [6.2, 5.6, 5.0]])    # G3: overlaps G0 heavily -> full/full ties
    rad_lu = np.array([3.2, 2.1, 2.6, 2.4])
    pos = (xc - 0.5) * dx + xmin
    return pos, rad_lu * dx


def scen_psc():
    """PSCLattice3D collide (psclattice3d.py:187-358) + stream, physical units."""
    rng = np.random.default_rng(13)
    nx, ny, nz = 14, 12, 10
    dx, dt, rho_phys = 1e-3, 2e-4, 1000.0
    xmin = np.array([0.0, 0.0, 0.0])
    pos, rad = _psc_particles(dx, xmin)
    n = len(rad)
    vel = 1e-3 * rng.uniform(-1, 1, (n, 3))
    omg = 0.5 * rng.uniform(-1, 1, (n, 3))
    domain = (0.0, (nx - 2) * dx, 0.0, (ny - 2) * dx, 0.0, (nz - 2) * dx)
    dem = make_dem(domain, dt / 5, (0, 0, -9.81), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2500.0, pos, vel, omega=omg)
    lat = PSCLattice3D(nx, ny, nz, 1.0 / 0.65, dx, dt, rho_phys, dem)
    set_walls_z(lat)
    random_flow(lat, rng, 0.01, 0.002)
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy(),
                gpos=pos, grad=rad, gvel=vel, gomega=omg, dx=dx, dt=dt, rho_unit=rho_phys,
                domain=np.array(domain))
    lat.initialize()
    out = dict(id_init=lat.id.to_numpy(), volfrac_init=lat.volfrac.to_numpy(),
               weight_init=lat.weight.to_numpy(), velsolid_init=lat.velsolid.to_numpy())
    for s in range(3):
        lat.collide()
        for k in ("id", "volfrac", "weight", "velsolid", "hydroforce"):
            out[f"{k}_{s}"] = getattr(lat, k).to_numpy()
        out[f"force_fluid_{s}"] = dem.gf.force_fluid.to_numpy()
        out[f"moment_fluid_{s}"] = dem.gf.moment_fluid.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("psc", omega0=np.float64(1.0 / 0.65), nsteps=np.int64(3), **init, **out)


def scen_hybrid():
    """HybridLattice3D with coarse grains only = PSC + Smagorinsky
    (hybridlattice.py:433-503), lattice units."""
    rng = np.random.default_rng(14)
    nx, ny, nz = 14, 12, 10
    dx = dt = rho_phys = 1.0
    xmin = np.zeros(3)
    pos, rad = _psc_particles(dx, xmin)
    n = len(rad)
    vel = 2e-3 * rng.uniform(-1, 1, (n, 3))
    omg = 1e-3 * rng.uniform(-1, 1, (n, 3))
    domain = (0.0, nx - 2.0, 0.0, ny - 2.0, 0.0, nz - 2.0)
    dem = make_dem(domain, 0.1, (0, 0, -1e-5), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2.5, pos, vel, omega=omg)
    lat = HybridLattice3D(nx, ny, nz, 1.0 / 0.6, dx, dt, rho_phys, dem)
    set_walls_z(lat)
    random_flow(lat, rng, 0.04, 0.005)
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy(),
                gpos=pos, grad=rad, gvel=vel, gomega=omg, domain=np.array(domain))
    lat.initialize_complete()
    out = {}
    for s in range(3):
        lat.prepare_step()
        lat.collide()
        out[f"omega_{s}"] = lat.omega.to_numpy()
        out[f"weight_{s}"] = lat.coarse_weight.to_numpy()
        out[f"id_{s}"] = lat.coarse_id.to_numpy()
        out[f"volfrac_{s}"] = lat.coarse_volfrac.to_numpy()
        out[f"hydroforce_{s}"] = lat.hydroforce.to_numpy()
        lat.stream()
        lat.lattice2grains()
        out[f"force_fluid_{s}"] = dem.gf.force_fluid.to_numpy()
        out[f"moment_fluid_{s}"] = dem.gf.moment_fluid.to_numpy()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("hybrid", omega0=np.float64(1.0 / 0.6), cs=np.float64(BasicLattice3D.SmagorinskyConstant),
         nsteps=np.int64(3), **init, **out)


def _dem_particles(rng):
    """12 spheres in a 40x30x30 box: approaching pairs, an initially overlapping
    pair, wall contacts, and one pair that touches only across the periodic x
    boundary (never proposed by the reference broad phase)."""
    pos = np.array([
        [10.0, 10.0, 10.0], [14.9, 10.2, 10.1],    # approaching pair
        [20.0, 20.0, 6.0], [24.4, 20.5, 6.4],      # overlapping pair
        [30.0, 8.0, 2.52],                         # on the z=0 wall
        [5.0, 27.4, 15.0],                         # near y=max wall
        [1.2, 15.0, 20.0], [38.6, 15.1, 20.2],     # touching across periodic x
        [15.0, 20.0, 20.0], [15.0, 24.7, 20.3],    # approaching pair (y)
        [30.0, 22.0, 22.0], [34.6, 22.0, 26.0],
    ])
    rad = np.array([2.5, 2.4, 2.2, 2.3, 2.5, 2.6, 1.8, 1.9, 2.4, 2.3, 2.0, 2.7])
    vel = 0.02 * rng.uniform(-1, 1, (12, 3))
    vel[0] = [0.05, 0.0, 0.0]
    vel[1] = [-0.05, 0.0, 0.0]
    vel[4] = [0.0, 0.0, -0.03]
    vel[5] = [0.0, 0.04, 0.0]
    vel[8] = [0.0, 0.04, 0.01]
    vel[9] = [0.0, -0.04, 0.0]
    omg = 0.05 * rng.uniform(-1, 1, (12, 3))
    return pos, rad, vel, omg


def _scen_dem(name, contact, model, seed):
    rng = np.random.default_rng(seed)
    pos, rad, vel, omg = _dem_particles(rng)
    domain = (0.0, 40.0, 0.0, 30.0, 0.0, 30.0)
    dem = make_dem(domain, 0.05, (0.0, 0.0, -2e-3), contact, rad, 2.0, pos, vel, omega=omg,
                   periodic=(True, False, False), E=1e3, nu=0.3, wall_E=2e3, wall_nu=0.25,
                   model=model)
    ff = 1e-3 * rng.uniform(-1, 1, (12, 3))
    mf = 1e-3 * rng.uniform(-1, 1, (12, 3))
    dem.gf.force_fluid.from_numpy(ff)
    dem.gf.moment_fluid.from_numpy(mf)
    init = dict(gpos=pos, grad=rad, gvel=vel, gomega=omg, force_fluid=ff, moment_fluid=mf,
                domain=np.array(domain), dt=0.05, gravity=np.array([0.0, 0.0, -2e-3]),
                periodic=np.array([1, 0, 0]), density=2.0, E=1e3, nu=0.3, wall_E=2e3, wall_nu=0.25,
                max_coord=16, mass=dem.gf.mass.to_numpy(), table_size=dem.bpcd.hash_table.shape[0],
                cell_size=dem.bpcd.cell_size)
    out = {}
    nsub = 60
    for s in range(nsub):
        dem.run_simulation()
        if (s + 1) % 5 == 0:
            st = dem_state(dem)
            for k, v in st.items():
                out[f"{k}_{s + 1}"] = v
            pairs, shear, wact, wshear = dem_contacts(dem)
            out[f"pairs_{s + 1}"] = pairs
            out[f"shear_{s + 1}"] = shear
            out[f"wact_{s + 1}"] = wact
            out[f"wshear_{s + 1}"] = wshear
    save(name, nsub=np.int64(nsub), **init, **out)


def scen_dem_hertz():
    _scen_dem("dem_hertz", HertzContactConfig(pp_friction=0.3, pw_friction=0.4,
                                              pp_restitution=0.9, pw_restitution=0.8), "hertz", 21)


def scen_dem_linear():
    _scen_dem("dem_linear", LinearContactConfig(stiffness_normal=200.0, stiffness_tangential=100.0,
                                                damping_normal=0.2, damping_tangential=0.1,
                                                pp_friction=0.3, pw_friction=0.4), "linear", 22)


def scen_coupled():
    """Driver loop of single_particle_settle.py:230-241 (collide, stream,
    DEM x subCycles) on a small box, lattice units, two spheres near the floor."""
    rng = np.random.default_rng(31)
    nx, ny, nz = 12, 12, 16
    pos = np.array([[5.5, 5.6, 3.4], [6.1, 6.0, 9.2]])   # physical = lattice - 0.5 at xmin=0
    rad = np.array([3.0, 2.6])
    vel = np.array([[0.0, 0.0, -0.01], [0.002, 0.0, -0.02]])
    omg = 1e-3 * rng.uniform(-1, 1, (2, 3))
    domain = (0.0, nx - 2.0, 0.0, ny - 2.0, 0.0, nz - 2.0)
    sub = 4
    dem = make_dem(domain, 1.0 / sub, (0.0, 0.0, -1e-4), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2.5, pos, vel, omega=omg, periodic=(True, True, False))
    lat = PSCLattice3D(nx, ny, nz, 1.0 / 0.6, 1.0, 1.0, 1.0, dem)
    set_walls_z(lat)
    init = dict(ct=lat.CT.to_numpy(), gpos=pos, grad=rad, gvel=vel, gomega=omg,
                domain=np.array(domain), sub=np.int64(sub), dt_dem=1.0 / sub,
                gravity=np.array([0.0, 0.0, -1e-4]), density=2.5)
    lat.initialize()
    out = {}
    nsteps = 4
    for s in range(nsteps):
        lat.collide()
        lat.stream()
        for _ in range(sub):
            dem.run_simulation()
        for k, v in dem_state(dem).items():
            out[f"{k}_{s}"] = v
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
        out[f"id_{s}"] = lat.id.to_numpy()
    out["f_last"] = lat.f.to_numpy()
    save("coupled", omega0=np.float64(1.0 / 0.6), nsteps=np.int64(nsteps), **init, **out)


def scen_couette_ladd():
    """PSCLattice3D between two moving walls (VEL_LADD cells, the modified
    bounce-back of lbm_solver3d.py:222-225, as in the shear-suspension
    driver shear_fullyresolved.py:36-45) with one sphere, lattice units."""
    rng = np.random.default_rng(41)
    nx, ny, nz = 12, 10, 12
    U = 0.02
    pos = np.array([[5.6, 4.7, 5.3]])
    rad = np.array([2.4])
    vel = np.array([[0.001, 0.0, 0.0]])
    omg = np.array([[0.0, 0.002, 0.0]])
    domain = (0.0, float(nx), 0.0, float(ny), 0.0, float(nz))
    dem = make_dem(domain, 0.25, (0.0, 0.0, 0.0), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2.0, pos, vel, omega=omg, periodic=(True, True, False))
    lat = PSCLattice3D(nx, ny, nz, 1.0 / 0.7, 1.0, 1.0, 1.0, dem)
    ct = lat.CT.arr
    ct[:, :, 0] = CellType.VEL_LADD
    ct[:, :, -1] = CellType.VEL_LADD
    random_flow(lat, rng, 0.01, 0.003)
    lat.vel.arr[:, :, 0, :] = (-U, 0.0, 0.0)
    lat.vel.arr[:, :, -1, :] = (U, 0.005, 0.0)
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy(),
                gpos=pos, grad=rad, gvel=vel, gomega=omg, domain=np.array(domain))
    lat.initialize()
    out = {}
    for s in range(3):
        lat.collide()
        out[f"force_fluid_{s}"] = dem.gf.force_fluid.to_numpy()
        out[f"moment_fluid_{s}"] = dem.gf.moment_fluid.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
        # stress diagnostics of the shear driver (lbm_solver3d.py:347-456)
        lat.compute_stress()
        for k in ("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz",
                  "shear_stress_mag"):
            out[f"{k}_{s}"] = getattr(lat, k).to_numpy()
        out[f"plane_top_{s}"] = np.asarray(lat.compute_plane_average_stress(2, nz - 2), np.float64)
        out[f"plane_y_{s}"] = np.asarray(lat.compute_plane_average_stress(1, 3), np.float64)
        out[f"plane_x_{s}"] = np.asarray(lat.compute_plane_average_stress(0, 4), np.float64)
    save("couette_ladd", omega0=np.float64(1.0 / 0.7), nsteps=np.int64(3), **init, **out)


def _scen_open(name, axis, low, high, U, seed):
    """PSCLattice3D with open boundaries on the two faces normal to `axis`:
    `low` / `high` are (CellType bits, value) -- VEL_INLET_LADD and VEL_ZOUHE
    take a velocity along the axis, Pre_ZOUHE a density (wet-node and Ladd-inlet
    rules of lbm_solver3d.py:216-250, 516-527, 671-962); the other axes are
    periodic; one sphere; lattice units."""
    rng = np.random.default_rng(seed)
    shape = [10, 9, 8]
    shape[axis] = 14
    nx, ny, nz = shape
    pos = np.array([[nx / 2 - 0.3, ny / 2 + 0.2, nz / 2 - 0.1]])
    rad = np.array([2.2])
    domain = (0.0, float(nx), 0.0, float(ny), 0.0, float(nz))
    per = [True, True, True]
    per[axis] = False
    dem = make_dem(domain, 0.25, (0.0, 0.0, 0.0), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2.0, pos, np.zeros((1, 3)), periodic=tuple(per))
    lat = PSCLattice3D(nx, ny, nz, 1.0 / 0.7, 1.0, 1.0, 1.0, dem)
    random_flow(lat, rng, 0.005, 0.002)
    ct = lat.CT.arr
    for (bits, val), idx in ((low, 0), (high, shape[axis] - 1)):
        sl = [slice(None)] * 3
        sl[axis] = idx
        sl = tuple(sl)
        ct[sl] = bits
        if bits & CellType.Pre_ZOUHE:
            lat.rho.arr[sl] = val
            lat.vel.arr[sl] = 0.0
        else:
            v = np.zeros(3)
            v[axis] = val
            lat.vel.arr[sl] = v
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy(),
                gpos=pos, grad=rad, gvel=np.zeros((1, 3)), gomega=np.zeros((1, 3)), domain=np.array(domain),
                periodic=np.array(per))
    lat.initialize()
    out = {}
    for s in range(4):
        lat.collide()
        out[f"force_fluid_{s}"] = dem.gf.force_fluid.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save(name, omega0=np.float64(1.0 / 0.7), nsteps=np.int64(4), **init, **out)


def scen_open_x():
    """The packed-bed pressure-drop driver's boundaries (pressure_drop_fully.py:106-116):
    Ladd velocity inlet at x = 0, Zou-He pressure outlet at x = Nx-1."""
    _scen_open("open_x", 0, (CellType.VEL_INLET_LADD | CellType.LEFT, 0.02),
               (CellType.Pre_ZOUHE | CellType.RIGHT, 1.0), 0.02, 51)


def scen_open_y():
    """Zou-He velocity inlet at y = 0, Zou-He pressure outlet at y = Ny-1."""
    _scen_open("open_y", 1, (CellType.VEL_ZOUHE | CellType.BOTTOM, 0.015),
               (CellType.Pre_ZOUHE | CellType.TOP, 0.998), 0.015, 52)


def scen_open_z():
    """Zou-He pressure at z = 0, Ladd velocity inlet at z = Nz-1 (flow towards -z)."""
    _scen_open("open_z", 2, (CellType.Pre_ZOUHE | CellType.BACK, 1.001),
               (CellType.VEL_INLET_LADD | CellType.FRONT, -0.02), -0.02, 53)


def scen_open_xr():
    """Zou-He pressure at x = 0, Zou-He velocity inlet at x = Nx-1 (flow towards -x)."""
    _scen_open("open_xr", 0, (CellType.Pre_ZOUHE | CellType.LEFT, 1.0),
               (CellType.VEL_ZOUHE | CellType.RIGHT, -0.018), -0.018, 54)


def scen_open_exit_x():
    """Zou-He velocity inlet at x = 0, convective exit (VEL_EXIT) at x = Nx-1."""
    _scen_open("open_exit_x", 0, (CellType.VEL_ZOUHE | CellType.LEFT, 0.02),
               (CellType.VEL_EXIT | CellType.RIGHT, 0.0), 0.02, 55)


def scen_open_exit_z():
    """Convective exit at z = 0, Zou-He velocity inlet at z = Nz-1 (flow towards -z)."""
    _scen_open("open_exit_z", 2, (CellType.VEL_EXIT | CellType.BACK, 0.0),
               (CellType.VEL_ZOUHE | CellType.FRONT, -0.02), -0.02, 56)


def scen_open_yr():
    """Zou-He pressure at y = 0, Zou-He velocity at y = Ny-1."""
    _scen_open("open_yr", 1, (CellType.Pre_ZOUHE | CellType.BOTTOM, 1.002),
               (CellType.VEL_ZOUHE | CellType.TOP, 0.015), 0.015, 57)


def scen_open_zb():
    """Zou-He velocity at z = 0, Zou-He pressure at z = Nz-1."""
    _scen_open("open_zb", 2, (CellType.VEL_ZOUHE | CellType.BACK, 0.02),
               (CellType.Pre_ZOUHE | CellType.FRONT, 1.0), 0.02, 58)


def scen_open_slip():
    """The pressure-drop channel with free-slip side walls: Ladd inlet at
    x = 0, Zou-He pressure at x = Nx-1, FREE_SLIP walls at y = 0 / Ny-1 set
    last (they own the corner cells), one PSC sphere (lbm_solver3d.py:230-236)."""
    rng = np.random.default_rng(59)
    nx, ny, nz = 14, 10, 8
    pos = np.array([[nx / 2 - 0.3, ny / 2 + 0.2, nz / 2 - 0.1]])
    rad = np.array([2.2])
    domain = (0.0, float(nx), 0.0, float(ny), 0.0, float(nz))
    dem = make_dem(domain, 0.25, (0.0, 0.0, 0.0), HertzContactConfig(0.3, 0.3, 0.9, 0.9),
                   rad, 2.0, pos, np.zeros((1, 3)), periodic=(False, False, True))
    lat = PSCLattice3D(nx, ny, nz, 1.0 / 0.7, 1.0, 1.0, 1.0, dem)
    random_flow(lat, rng, 0.005, 0.002)
    ct = lat.CT.arr
    ct[0] = CellType.VEL_INLET_LADD | CellType.LEFT
    lat.vel.arr[0] = (0.02, 0.0, 0.0)
    ct[-1] = CellType.Pre_ZOUHE | CellType.RIGHT
    lat.rho.arr[-1] = 1.0
    lat.vel.arr[-1] = 0.0
    ct[:, 0] = CellType.FREE_SLIP | CellType.BOTTOM
    ct[:, -1] = CellType.FREE_SLIP | CellType.TOP
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy(),
                gpos=pos, grad=rad, gvel=np.zeros((1, 3)), gomega=np.zeros((1, 3)), domain=np.array(domain))
    lat.initialize()
    out = {}
    for s in range(4):
        lat.collide()
        out[f"force_fluid_{s}"] = dem.gf.force_fluid.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("open_slip", omega0=np.float64(1.0 / 0.7), nsteps=np.int64(4), **init, **out)


def scen_open_smag():
    """BasicLattice3D (Smagorinsky, inlets skipped by initialize/collide) with a
    Ladd inlet at x = 0, a convective exit at x = Nx-1 and FREE_SLIP walls at
    z = 0 / Nz-1: the exit's equilibrium overwrite feeds the next computeOmega
    (lbm_solver3d.py:176-192, 645-663)."""
    rng = np.random.default_rng(60)
    nx, ny, nz = 14, 8, 9
    lat = BasicLattice3D(nx, ny, nz, 1.0 / 0.55, 1.0, 1.0, 1.0)
    random_flow(lat, rng, 0.03, 0.004)
    ct = lat.CT.arr
    ct[0] = CellType.VEL_INLET_LADD | CellType.LEFT
    lat.vel.arr[0] = (0.04, 0.0, 0.0)
    ct[-1] = CellType.VEL_EXIT | CellType.RIGHT
    ct[:, :, 0] = CellType.FREE_SLIP | CellType.BACK
    ct[:, :, -1] = CellType.FREE_SLIP | CellType.FRONT
    init = dict(ct=lat.CT.to_numpy(), rho0=lat.rho.to_numpy(), vel0=lat.vel.to_numpy())
    lat.initialize()
    out = {}
    for s in range(4):
        lat.collide()
        out[f"omega_{s}"] = lat.omega.to_numpy()
        lat.stream()
        out[f"f_{s}"] = lat.f.to_numpy()
        out[f"rho_{s}"] = lat.rho.to_numpy()
        out[f"vel_{s}"] = lat.vel.to_numpy()
    save("open_smag", omega0=np.float64(1.0 / 0.55), cs=np.float64(BasicLattice3D.SmagorinskyConstant),
         nsteps=np.int64(4), **init, **out)


def scen_p4io():
    """DEMSolver.save_single (demsolver.py:59-128) after 20 sub-steps of the
    DEM scenario: the text of one p4p and one p4c frame and the arrays it was
    written from (the active contacts in the reference's slot order)."""
    import io
    rng = np.random.default_rng(21)
    pos, rad, vel, omg = _dem_particles(rng)
    domain = (0.0, 40.0, 0.0, 30.0, 0.0, 30.0)
    dem = make_dem(domain, 0.05, (0.0, 0.0, -2e-3),
                   HertzContactConfig(pp_friction=0.3, pw_friction=0.4, pp_restitution=0.9, pw_restitution=0.8),
                   rad, 2.0, pos, vel, omega=omg, periodic=(True, False, False), E=1e3, nu=0.3, wall_E=2e3,
                   wall_nu=0.25, model="hertz")
    for _ in range(20):
        dem.run_simulation()
    p4p, p4c = io.StringIO(), io.StringIO()
    t = 1.25
    dem.save_single(p4p, p4c, t)
    cf = dem.cf
    act = cf.isActive.to_numpy().astype(bool)
    gf = dem.gf
    save("p4io", p4p=np.array(p4p.getvalue()), p4c=np.array(p4c.getvalue()), t=np.float64(t),
         ID=gf.ID.to_numpy(), group=gf.groupID.to_numpy(), radius=gf.radius.to_numpy(), mass=gf.mass.to_numpy(),
         position=gf.position.to_numpy(), velocity=gf.velocity.to_numpy(), ci=cf.i.to_numpy()[act],
         cj=cf.j.to_numpy()[act], cpos=cf.position.to_numpy()[act], cforce=cf.force_a.to_numpy()[act])


def scen_host_api():
    """Host-side helpers drivers use (lbmutils.py:14-63, demconfig.py,
    types.py, contact_model.py): UnitConverter conversions, the configuration
    state after the setters, summary() text, and which inputs raise."""
    from src.lbm3d.lbmutils import UnitConverter
    uc = UnitConverter(2e-3, 1e-4, 1000.0)
    names = [m for m in dir(UnitConverter) if m.startswith(("getLb", "getPhys"))]
    conv = np.array([[getattr(uc, m)(v) for v in (0.5, 3.0)] for m in names])
    cfg = DEMSolverConfig(domain=DomainBounds(0.0, 1.0, 0.0, 2.0, -1.0, 3.0), dt=1e-4,
                          gravity=Vector3(0.0, 0.0, -9.81),
                          contact_model=HertzContactConfig(pp_friction=0.3, pw_friction=0.4, pp_restitution=0.9,
                                                           pw_restitution=0.8))
    cfg.set_particle_properties(elastic_modulus=1e6, poisson_ratio=0.25, density=2650.0, max_coordinate_number=12)
    cfg.set_wall_properties(density=2500.0, elastic_modulus=2e6, poisson_ratio=0.3)
    cfg.set_periodic_boundaries(True, False, True)
    cfg.update_contact_model(pp_friction=0.5)
    lin = DEMSolverConfig(domain=DomainBounds(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), dt=2e-4, gravity=Vector3(0.0, -1.0, 0.0),
                          contact_model=LinearContactConfig(stiffness_normal=1e5, stiffness_tangential=5e4,
                                                            damping_normal=0.1, damping_tangential=0.05,
                                                            pp_friction=0.2, pw_friction=0.3))

    def raises(fn):
        try:
            fn()
        except ValueError:
            return True
        return False

    bad = np.array([
        raises(lambda: DomainBounds(1.0, 0.0, 0.0, 1.0, 0.0, 1.0)),
        raises(lambda: DEMSolverConfig(DomainBounds(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), 0.0, Vector3(0.0, 0.0, 0.0),
                                       HertzContactConfig(0.3, 0.3, 0.9, 0.9))),
        raises(lambda: cfg.set_particle_properties(bogus=1.0)),
        raises(lambda: cfg.set_wall_properties(bogus=1.0)),
        raises(lambda: cfg.update_contact_model(bogus=1.0)),
        raises(lambda: HertzContactConfig(1.5, 0.3, 0.9, 0.9).validate()),
        raises(lambda: HertzContactConfig(0.3, 0.3, 1.2, 0.9).validate()),
        raises(lambda: LinearContactConfig(-1.0, 1.0, 0.1, 0.1, 0.3, 0.3).validate()),
        raises(lambda: LinearContactConfig(1.0, 1.0, -0.1, 0.1, 0.3, 0.3).validate()),
        raises(lambda: LinearContactConfig(1.0, 1.0, 0.1, 0.1, 0.3, 1.3).validate()),
    ])
    pp, wp = cfg.particle_props, cfg.wall_props
    save("host_api", conv_names=np.array(names), conv=conv, boundary_type=np.array(cfg.boundaryType),
         wall_normals=np.array([np.asarray(v, float) for v in cfg.wall_normals]),
         wall_distances=np.array(cfg.wall_distances, float), domain_min=np.asarray(cfg.domain_min, float),
         domain_max=np.asarray(cfg.domain_max, float),
         particle_props=np.array([pp.elastic_modulus, pp.poisson_ratio, pp.density, pp.max_coordinate_number], float),
         wall_props=np.array([wp.density, wp.elastic_modulus, wp.poisson_ratio], float),
         pp_friction=np.float64(cfg.contact_model.pp_friction), summary_hertz=np.array(cfg.summary()),
         summary_linear=np.array(lin.summary()), raises=bad)


SCENARIOS = {
    "bgk_smag": scen_bgk_smag, "forced": scen_forced, "psc": scen_psc, "hybrid": scen_hybrid,
    "dem_hertz": scen_dem_hertz, "dem_linear": scen_dem_linear, "coupled": scen_coupled,
    "couette_ladd": scen_couette_ladd, "open_x": scen_open_x, "open_y": scen_open_y, "open_z": scen_open_z,
    "open_xr": scen_open_xr, "open_exit_x": scen_open_exit_x, "open_exit_z": scen_open_exit_z,
    "open_yr": scen_open_yr, "open_zb": scen_open_zb, "open_slip": scen_open_slip, "open_smag": scen_open_smag,
    "p4io": scen_p4io, "host_api": scen_host_api,
}

if __name__ == "__main__":
    names = sys.argv[2:] or list(SCENARIOS)
    for nm in names:
        SCENARIOS[nm]()
