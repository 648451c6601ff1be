"""Open boundaries on the GPU (the boundary pass after the fused step):
Zou-He velocity / pressure on all six faces, convective exits, Ladd velocity
inlets and free-slip walls (lbm_solver3d.py:207-250, 516-527, 645-960),
against golden vectors from the reference's own source, and against the FP64
oracle on a larger packed-bed channel with the pressure-drop driver's
boundaries (pressure_drop_fully.py:106-116).

Every golden case runs twice: reading the fields after every step (the stream
goes through lbdem_stream_moments and its boundary pass, the next step reads
post-stream populations in place) and reading only at the end (the stream
happens inside the fused step and its boundary pass).

Tolerances (FP32 storage, FP32 arithmetic, against FP64):
  populations and density: absolute 1e-6 after four steps
  velocity: max error / max |u| <= 2e-5
  particle force: max error / max magnitude <= 1e-4
  omega (Smagorinsky): absolute 1e-6
  FP16 storage: density absolute 5e-5, total |drag| within 1e-3
  oracle channel (40 steps): populations absolute 2e-6, forces 2e-4, pressure drop 1e-4 relative
"""
import numpy as np
import pytest

from oracle.oracle import OracleGrains, OracleLattice
from tests.golden_util import load, relmax
from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu

OPEN = ("open_x", "open_y", "open_z", "open_xr", "open_exit_x", "open_exit_z", "open_yr", "open_zb", "open_slip")
OBST, FREE_SLIP, VEL_LADD, INLET = 8, 16, 32, 262144
LEFT, RIGHT, PRE_ZOUHE = 8192, 4096, 256


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)


def _psc(g, storage="f32"):
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    nx, ny, nz = g["ct"].shape
    rad = g["grad"]
    dem = make_dem(g["domain"], 0.25, (0, 0, 0), _hertz(), rad, 2.0 * 4.0 / 3.0 * np.pi * rad ** 3, g["gpos"],
                   g["gvel"], omega=g["gomega"])
    lat = PSCLattice3D(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem, storage=storage)
    lat.CT.from_numpy(g["ct"])
    lat.rho.from_numpy(g["rho0"])
    lat.vel.from_numpy(g["vel0"])
    return lat, dem


@pytest.mark.parametrize("read_every_step", [True, False])
@pytest.mark.parametrize("name", OPEN)
def test_open_boundaries_golden(name, read_every_step):
    g = load(name)
    lat, dem = _psc(g)
    lat.initialize()
    assert lat.has_open_boundaries
    skip = (g["ct"] & (OBST | FREE_SLIP | VEL_LADD)) != 0   # never initialised by the reference
    n = int(g["nsteps"])
    for s in range(n):
        lat.collide()
        assert relmax(dem.gf.force_fluid.to_numpy(), g[f"force_fluid_{s}"]) < 1e-4
        lat.stream()
        if read_every_step or s == n - 1:
            assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[~skip].max() < 1e-6
            assert np.abs(lat.rho.to_numpy() - g[f"rho_{s}"]).max() < 1e-6
            assert relmax(lat.vel.to_numpy(), g[f"vel_{s}"]) < 2e-5
    lat.check_status()


@pytest.mark.parametrize("read_every_step", [True, False])
def test_open_boundaries_smagorinsky_golden(read_every_step):
    """BasicLattice3D (Smagorinsky; the inlet is skipped by initialize/collide):
    Ladd inlet, convective exit, free-slip walls."""
    from lbdem_taichi_b200.lbm3d.lattice import BasicLattice3D
    g = load("open_smag")
    nx, ny, nz = g["ct"].shape
    lat = BasicLattice3D(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0)
    lat.CT.from_numpy(g["ct"])
    lat.rho.from_numpy(g["rho0"])
    lat.vel.from_numpy(g["vel0"])
    lat.initialize()
    skip = (g["ct"] & (OBST | FREE_SLIP | VEL_LADD | INLET)) != 0
    n = int(g["nsteps"])
    for s in range(n):
        lat.collide()
        if read_every_step or s == n - 1:
            assert np.abs(lat.omega.to_numpy() - g[f"omega_{s}"])[~skip].max() < 1e-6
        lat.stream()
        if read_every_step or s == n - 1:
            assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[~skip].max() < 1e-6
            assert np.abs(lat.rho.to_numpy() - g[f"rho_{s}"]).max() < 1e-6
            assert relmax(lat.vel.to_numpy(), g[f"vel_{s}"]) < 2e-5
    lat.check_status()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_open_boundaries_16bit_storage(storage):
    """16-bit population storage through the boundary pass: density and the
    total drag of the inlet / pressure-outlet case against the golden."""
    g = load("open_x")
    lat, dem = _psc(g, storage=storage)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.collide()
        lat.stream()
    F = dem.gf.force_fluid.to_numpy()
    ref = g["force_fluid_3"]
    drho = np.abs(lat.rho.to_numpy() - g["rho_3"]).max()
    tol = 5e-5 if storage == "f16" else 2e-3
    assert drho < tol, drho
    ftol = 1e-3 if storage == "f16" else 2e-2
    assert np.abs(F - ref).sum() <= ftol * np.abs(ref).sum(), (F, ref)
    lat.check_status()


def test_pressure_drop_channel_vs_oracle():
    """Packed-bed channel with the pressure-drop driver's boundaries: Ladd
    velocity inlet at x = 0, Zou-He pressure outlet (rho = 1) at x = Nx-1,
    periodic in y and z, 14 spheres; 40 steps through the fused kernel and the
    boundary pass against the FP64 oracle, then the pressure drop between the
    planes at 0.1 and 0.9 of the length (the driver's sampling planes)."""
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    rng = np.random.default_rng(77)
    nx, ny, nz = 96, 40, 36
    pos, rad = rsa_spheres(rng, 14, (nx - 30, ny, nz), 7.0, 10.0, gap=1.0, margin=1.0)
    pos[:, 0] += 15.0
    n = len(rad)
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    domain = (0.0, float(nx), 0.0, float(ny), 0.0, float(nz))
    dem = make_dem(domain, 0.1, (0, 0, 0), _hertz(), rad, mass, pos, np.zeros((n, 3)), periodic=(False, True, True))
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem)
    ct = np.full((nx, ny, nz), 1, np.int32)
    ct[0] = INLET | LEFT
    ct[-1] = PRE_ZOUHE | RIGHT
    u_in = 0.02
    vel = np.zeros((nx, ny, nz, 3))
    rho = np.ones((nx, ny, nz))
    # the driver's per-element form (pressure_drop_fully.py:111-116)
    lat.CT.from_numpy(ct)
    for j in range(ny):
        for k in range(nz):
            lat.vel[0, j, k][0] = u_in
            lat.rho[nx - 1, j, k] = 1.0
    vel[0, :, :, 0] = u_in
    np.testing.assert_array_equal(lat.vel.to_numpy(), vel)
    o = OracleLattice(nx, ny, nz, 1 / 0.6, psc=True)
    o.ct[...] = ct
    o.vel[...] = vel
    o.rho[...] = rho
    og = OracleGrains(pos, rad, np.zeros((n, 3)), np.zeros((n, 3)))
    lat.initialize()
    o.initialize()
    for _ in range(40):
        lat.collide()
        lat.stream()
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        o.stream()
    assert np.abs(lat.f.to_numpy() - o.f).max() < 2e-6
    r = lat.rho.to_numpy()
    assert np.abs(r - o.rho).max() < 2e-6
    assert relmax(lat.vel.to_numpy(), o.vel) < 5e-5
    assert relmax(dem.gf.force_fluid.to_numpy(), og.force_fluid) < 2e-4
    i0, i1 = int(0.1 * nx), int(0.9 * nx)
    dp = (r[i0].mean() - r[i1].mean()) / 3.0
    dpo = (o.rho[i0].mean() - o.rho[i1].mean()) / 3.0
    assert dpo > 0 and abs(dp - dpo) <= 1e-4 * dpo, (dp, dpo)
    lat.check_status()


def test_boundary_list_and_launch_count():
    """The boundary pass lists exactly the wet-node cells (first pass: Zou-He;
    second pass: exits and inlets) and adds one launch per non-empty pass."""
    from lbdem_taichi_b200 import _native as N
    g = load("open_x")
    lat, _ = _psc(g)
    lat.initialize()
    nx, ny, nz = g["ct"].shape
    assert (lat._lat.bnd_na, lat._lat.bnd_nb) == (ny * nz, ny * nz)
    cells = lat._bnd[: ny * nz * 2].cpu().numpy()
    x = cells % nx
    assert (x[: ny * nz] == nx - 1).all() and (x[ny * nz:] == 0).all()
    assert (np.diff(cells[: ny * nz]) > 0).all() and (np.diff(cells[ny * nz:]) > 0).all()
    N.reset_launch_count()
    lat.collide()
    lat.stream()
    lat.collide()
    # map (clear + scatter) + step (1) + two boundary passes, twice
    assert N.launch_count() == 2 * (2 + 1 + 2)
