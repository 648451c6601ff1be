"""GPU path vs the FP64 oracle on seeded inputs larger than the golden cases.

Tolerances:
  owner id and solid-fraction sub-cell counts: exact
  FP32 populations: absolute 2e-6 after 10 steps (deviation storage)
  particle force / torque: max error / max magnitude <= 2e-4
  DEM (FP64 both sides): positions absolute 1e-9, contact sets exact
  FP16 storage: total drag error <= 1e-3 of the drag scale (sum of |F_i|) vs FP64
  every step, per-particle drag <= 1e-2; BF16 2e-2 / 1e-1
"""
import numpy as np
import pytest

from oracle.oracle import OracleDEM, OracleGrains, OracleLattice
from tests.golden_util import relmax
from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu

OBST, FLUID = 8, 1


def _ct_zwalls(nx, ny, nz):
    ct = np.full((nx, ny, nz), FLUID, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = OBST
    return ct


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)


def _pair(nx, ny, nz, pos, rad, vel, omega, *, dx=1.0, dt=1.0, rho_u=1.0, smag="reference", force=None,
          storage="f32", periodic=(True, True, False), dt_dem=0.1, gravity=(0, 0, 0), ct=None, max_coord=16):
    """(gpu lattice, gpu dem, oracle lattice, oracle dem, oracle grains) on the same inputs."""
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    domain = (0.0, nx * dx, 0.0, ny * dx, 0.0, nz * dx)
    dem = make_dem(domain, dt_dem, gravity, _hertz(), rad, mass, pos, vel, omega=omega, periodic=periodic,
                   max_coord=max_coord)
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, dx, dt, rho_u, dem, smagorinsky=smag, body_force=force,
                       storage=storage)
    ct = _ct_zwalls(nx, ny, nz) if ct is None else ct
    lat.CT.from_numpy(ct)
    o = OracleLattice(nx, ny, nz, 1 / 0.6, dx=dx, dt=dt, rho_unit=rho_u, smag=smag == "reference", psc=True,
                      force=force)
    o.ct[...] = ct
    od = OracleDEM(pos, vel, rad, mass, dt=dt_dem, gravity=gravity, domain=domain, periodic=periodic, E=1e5,
                   nu=0.3, wall_E=1e5, wall_nu=0.3, pp_mu=0.3, pw_mu=0.3, pp_e=0.9, pw_e=0.9,
                   max_coord=max_coord, omega=omega)
    og = OracleGrains(od.pos, od.radius, od.vel, od.omega)
    og.pos, og.vel, og.omega, og.force_fluid, og.moment_fluid = (od.pos, od.vel, od.omega, od.force_fluid,
                                                                 od.moment_fluid)
    return lat, dem, o, od, og


def test_map_exact_with_overlapping_spheres():
    """Winner rule with heavy overlap, partial/full covers, walls and spheres
    sticking out of the lattice: owner id and sub-cell count bit-exact."""
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    rng = np.random.default_rng(5)
    nx, ny, nz = 72, 64, 56
    n = 300
    dx = 1e-3
    pos = rng.uniform(-2.0, [nx + 2.0, ny + 2.0, nz + 2.0], (n, 3)) * dx
    rad = rng.uniform(1.0, 6.5, n) * dx
    vel = rng.normal(0, 1e-3, (n, 3)) * dx
    omg = rng.normal(0, 1e-3, (n, 3))
    mass = 2.0 * rad ** 3
    domain = (-10 * dx, (nx + 10) * dx, -10 * dx, (ny + 10) * dx, -10 * dx, (nz + 10) * dx)
    dem = make_dem(domain, 1e-3, (0, 0, 0), _hertz(), rad, mass, pos, vel, omega=omg)
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, dx, 2e-4, 1000.0, dem)
    ct = _ct_zwalls(nx, ny, nz)
    ct[10:20, 5:9, 30] = OBST
    lat.CT.from_numpy(ct)
    lat.initialize()
    o = OracleLattice(nx, ny, nz, 1 / 0.6, dx=dx, dt=2e-4, rho_unit=1000.0, psc=True,
                      dom_min=(domain[0], domain[2], domain[4]))
    o.ct[...] = ct
    og = OracleGrains(pos, rad, vel, omg)
    o.grains2lattice(og)
    np.testing.assert_array_equal(lat.id.to_numpy(), o.id)
    np.testing.assert_array_equal(np.rint(lat.volfrac.to_numpy() * 125).astype(int), np.rint(o.volfrac * 125).astype(int))
    assert relmax(lat.velsolid.to_numpy(), o.velsolid) < 1e-5
    assert (o.id >= 0).sum() > 10000


def test_fused_step_vs_oracle():
    rng = np.random.default_rng(7)
    nx, ny, nz = 64, 48, 40
    pos, rad = rsa_spheres(rng, 40, (nx, ny, nz), 6.0, 11.0, gap=1.0, margin=1.5)
    vel = rng.normal(0, 2e-3, (40, 3))
    omg = rng.normal(0, 2e-3, (40, 3))
    lat, dem, o, od, og = _pair(nx, ny, nz, pos, rad, vel, omg, force=(2e-6, -1e-6, 0.0))
    u0 = 0.02 * rng.uniform(-1, 1, (nx, ny, nz, 3))
    r0 = 1.0 + 0.002 * rng.uniform(-1, 1, (nx, ny, nz))
    lat.vel.from_numpy(u0)
    lat.rho.from_numpy(r0)
    o.vel[...] = u0
    o.rho[...] = r0
    lat.initialize()
    o.initialize()
    fl = o.ct == FLUID
    for s in range(10):
        lat.collide()
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        np.testing.assert_array_equal(lat.id.to_numpy(), o.id)
        assert relmax(dem.gf.force_fluid.to_numpy(), og.force_fluid) < 2e-4, s
        assert relmax(dem.gf.moment_fluid.to_numpy(), og.moment_fluid) < 2e-4, s
        lat.stream()
        o.stream()
    assert np.abs(lat.f.to_numpy() - o.f)[fl].max() < 2e-6
    assert relmax(lat.vel.to_numpy()[fl], o.vel[fl]) < 1e-4
    lat.check_status()


def test_coupled_vs_oracle():
    rng = np.random.default_rng(8)
    nx, ny, nz = 48, 48, 48
    pos, rad = rsa_spheres(rng, 30, (nx, ny, nz), 6.0, 10.0, gap=0.3, margin=2.0)
    vel = rng.normal(0, 5e-3, (30, 3))
    lat, dem, o, od, og = _pair(nx, ny, nz, pos, rad, vel, None, force=(0.0, 0.0, -1e-5), gravity=(0, 0, -1e-4),
                                dt_dem=0.2)
    lat.initialize()
    o.initialize()
    for s in range(12):
        lat.step(5)
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        o.stream()
        for _ in range(5):
            od.run_simulation()
    assert np.abs(dem.gf.position.to_numpy() - od.pos).max() < 1e-7
    assert relmax(dem.gf.velocity.to_numpy(), od.vel) < 1e-4
    assert relmax(dem.gf.force_fluid.to_numpy(), od.force_fluid) < 5e-4
    lat.check_status()
    dem.check_status()


def test_dem_contact_sets_vs_oracle():
    """Jittered cubic packing with initial overlaps (about three contacts per
    sphere): contact pair sets (with histories) identical to the oracle's."""
    rng = np.random.default_rng(9)
    g = np.stack(np.meshgrid(np.arange(10), np.arange(10), np.arange(6), indexing="ij"), -1).reshape(-1, 3)
    pos = 2.5 + g * 3.95 + rng.uniform(-0.05, 0.05, g.shape)
    n = len(pos)
    rad = 2.0 + rng.uniform(-0.02, 0.02, n)
    vel = rng.normal(0, 0.02, (n, 3))
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    domain = (0.0, 40.0, 0.0, 40.0, 0.0, 26.0)
    kw = dict(E=1e3, nu=0.3, wall_E=1e3, wall_nu=0.3)
    dem = make_dem(domain, 0.05, (0, 0, -1e-3), _hertz(), rad, mass, pos, vel, periodic=(True, True, False),
                   max_coord=24, **kw)
    od = OracleDEM(pos, vel, rad, mass, dt=0.05, gravity=(0, 0, -1e-3), domain=domain, periodic=(True, True, False),
                   pp_mu=0.3, pw_mu=0.3, pp_e=0.9, pw_e=0.9, max_coord=24, **kw)
    for s in range(1, 31):
        dem.run_simulation()
        od.run_simulation()
        if s % 5 == 0:
            mine = dem.active_contacts()
            ref = od.active_pairs()
            assert set(mine) == set(ref), s
            assert len(ref) > 300
            for k in ref:
                assert np.allclose(mine[k][2], ref[k], rtol=1e-7, atol=1e-12)
            assert np.abs(dem.gf.position.to_numpy() - od.pos).max() < 1e-9
    dem.check_status()
    assert od.status == 0


@pytest.mark.parametrize("storage,tol_total,tol_particle", [("f16", 1e-3, 1e-2), ("bf16", 2e-2, 1e-1)])
def test_storage_forms_drag_error(storage, tol_total, tol_particle):
    """16-bit population storage against the FP64 oracle with moving particles
    (the DEM runs 5 sub-steps per lattice step on both sides), 100 coupled
    steps: the error of the total drag vector of every step, relative to the
    drag scale sum_i |F_i| (the particles' random velocities make their drags
    cancel in the total), within the bound of its form (the metric's 1e-3 for
    FP16), and the per-particle drag (sum of |dF_i| over sum of |F_i|, so
    errors of different particles cannot cancel) within a looser bound at
    every tenth step."""
    rng = np.random.default_rng(10)
    nx, ny, nz = 64, 64, 64
    pos, rad = rsa_spheres(rng, 30, (nx, ny, nz), 8.0, 12.0, gap=1.0, margin=1.0)
    vel = rng.normal(0, 1e-3, (30, 3))
    lat, dem, o, od, og = _pair(nx, ny, nz, pos, rad, vel, None, force=(1e-5, 0, 0), storage=storage,
                                periodic=(True, True, True), ct=np.full((nx, ny, nz), FLUID, np.int32),
                                gravity=(1e-5, 0, 0), dt_dem=0.2)
    lat.initialize()
    o.initialize()
    moved = 0.0
    for s in range(1, 101):
        lat.collide()
        lat.stream()
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        o.stream()
        F = dem.gf.force_fluid.to_numpy()
        ref = og.force_fluid
        tot = np.linalg.norm(F.sum(0) - ref.sum(0)) / np.linalg.norm(ref, axis=1).sum()
        assert tot <= tol_total, (storage, s, tot)
        if s % 10 == 0:
            part = np.linalg.norm(F - ref, axis=1).sum() / np.linalg.norm(ref, axis=1).sum()
            assert part <= tol_particle, (storage, s, part)
        dem.run_substeps(5)
        for _ in range(5):
            od.run_simulation()
        moved = max(moved, float(np.abs(od.pos - pos).max()))
    assert moved > 0.05      # the particles moved (the map changed from step to step)
    lat.check_status()
    dem.check_status()


@pytest.mark.parametrize("storage,tol", [("f32", 2e-6), ("f16", 3e-4)])
def test_moving_walls_vs_oracle(storage, tol):
    """Sheared suspension between VEL_LADD walls moving +-U (the setup of the
    reference's shear_fullyresolved.py:36-45): 12 steps through the fused
    kernel, then populations (max abs error, FP32 / FP16 storage) and the
    particle forces against the FP64 oracle.  The drag is measured as the
    sum of |F_x| so that opposite forces of particles in the two shear
    directions do not cancel."""
    from oracle.oracle import CT_VEL_LADD
    rng = np.random.default_rng(21)
    nx, ny, nz = 32, 24, 20
    pos, rad = rsa_spheres(rng, 5, (nx, ny, nz), 5.0, 7.0, gap=1.0, margin=1.5)
    ct = np.full((nx, ny, nz), FLUID, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = CT_VEL_LADD
    lat, dem, o, od, og = _pair(nx, ny, nz, pos, rad, np.zeros((5, 3)), np.zeros((5, 3)), smag="off", ct=ct,
                                storage=storage)
    U = 0.03
    v0 = np.zeros((nx, ny, nz, 3))
    v0[:, :, 0, 0] = -U
    v0[:, :, -1, 0] = U
    lat.vel.from_numpy(v0)
    o.vel[...] = v0
    lat.initialize()
    o.initialize()
    for _ in range(12):
        lat.collide()
        lat.stream()
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        o.stream()
    fl = ct == FLUID
    assert np.abs(lat.f.to_numpy() - o.f)[fl].max() < tol
    F = dem.gf.force_fluid.to_numpy()
    if storage == "f32":
        assert relmax(F, og.force_fluid) < 2e-4
    else:
        # 16-bit storage: total drag (the quantity the storage forms are held to) within 1e-3,
        # every component within 2e-2 of the largest
        assert np.abs(F[:, 0] - og.force_fluid[:, 0]).sum() <= 1e-3 * np.abs(og.force_fluid[:, 0]).sum()
        assert relmax(F, og.force_fluid) < 2e-2
    # the walls drive the flow
    assert lat.vel.to_numpy()[:, :, -2, 0].mean() > 0.2 * U
    lat.check_status()


def test_mass_conservation_periodic():
    rng = np.random.default_rng(11)
    nx = ny = nz = 96
    pos, rad = rsa_spheres(rng, 60, (nx, ny, nz), 8.0, 12.0, gap=1.0, margin=1.0)
    vel = rng.normal(0, 1e-3, (60, 3))
    lat, dem, *_ = _pair(nx, ny, nz, pos, rad, vel, None, force=(1e-6, 0, 0), periodic=(True, True, True),
                         ct=np.full((nx, ny, nz), FLUID, np.int32))
    lat.initialize()
    m0 = lat.global_sums()[0]
    for _ in range(50):
        lat.step(10)
    m1 = lat.global_sums()[0]
    assert abs(m1 - m0) / m0 < 1e-6
    lat.check_status()
    dem.check_status()


def test_fault_flags_nan_and_overflow():
    import lbdem_taichi_b200._native as Nat
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    nx, ny, nz = 16, 16, 16
    # NaN in the initial velocity field -> LBDEM_ST_NAN after one collide
    pos = np.array([[8.0, 8.0, 8.0]])
    rad = np.array([2.5])
    dem = make_dem((0, 16, 0, 16, 0, 16), 0.1, (0, 0, 0), _hertz(), rad, 2 * rad ** 3, pos, np.zeros((1, 3)))
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem)
    v = np.zeros((nx, ny, nz, 3))
    v[3, 4, 5, 0] = np.nan
    lat.vel.from_numpy(v)
    lat.initialize()
    lat.collide()
    with pytest.raises(Nat.LbdemError, match="non-finite"):
        lat.check_status()
    # three mutually overlapping spheres with room for one contact each
    pos = np.array([[5.0, 5.0, 5.0], [6.0, 5.0, 5.0], [5.5, 6.0, 5.0]])
    rad = np.array([1.0, 1.0, 1.0])
    dem = make_dem((0, 10, 0, 10, 0, 10), 1e-3, (0, 0, 0), _hertz(), rad, np.ones(3), pos, np.zeros((3, 3)),
                   max_coord=1)
    dem.run_simulation()
    with pytest.raises(Nat.LbdemError, match="max_coordinate_number"):
        dem.check_status()
    # particle outside the broad-phase grid
    pos = np.array([[5.0, 5.0, 5.0], [500.0, 5.0, 5.0]])
    rad = np.array([1.0, 1.0])
    dem = make_dem((0, 10, 0, 10, 0, 10), 1e-3, (0, 0, 0), _hertz(), rad, np.ones(2), pos, np.zeros((2, 3)))
    dem.run_simulation()
    with pytest.raises(Nat.LbdemError, match="broad-phase grid"):
        dem.check_status()


def test_default_max_coordinate_number_flags_overflow():
    """The reference's default max_coordinate_number is 0 (types.py:42): the
    first contact has no slot; the library reports it instead of writing."""
    import lbdem_taichi_b200._native as Nat
    pos = np.array([[5.0, 5.0, 5.0], [6.5, 5.0, 5.0]])
    rad = np.array([1.0, 1.0])
    dem = make_dem((0, 10, 0, 10, 0, 10), 1e-3, (0, 0, 0), _hertz(), rad, np.ones(2), pos, np.zeros((2, 3)),
                   max_coord=0)
    dem.run_simulation()
    with pytest.raises(Nat.LbdemError):
        dem.check_status()


@pytest.mark.parametrize("mode", ["cooperative", "cluster"])
def test_dem_single_launch_kernels_match_split_kernels(mode, monkeypatch):
    """The single-launch DEM paths -- the default cooperative grid (grid
    barriers between phases) and the opt-in single cluster -- give the
    contact sets and states of two launches per sub-step (FP64; only the
    order of the atomic force sums differs)."""
    rng = np.random.default_rng(13)
    g = np.stack(np.meshgrid(np.arange(8), np.arange(8), np.arange(5), indexing="ij"), -1).reshape(-1, 3)
    pos = 2.5 + g * 3.95 + rng.uniform(-0.05, 0.05, g.shape)
    n = len(pos)
    rad = 2.0 + rng.uniform(-0.02, 0.02, n)
    vel = rng.normal(0, 0.02, (n, 3))
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    domain = (0.0, 32.0, 0.0, 32.0, 0.0, 22.0)
    res = []
    for m in (mode, "split"):
        if m == "cooperative":
            monkeypatch.delenv("LBDEM_DEM_KERNELS", raising=False)
        else:
            monkeypatch.setenv("LBDEM_DEM_KERNELS", m)
        dem = make_dem(domain, 0.05, (0, 0, -1e-3), _hertz(), rad, mass, pos, vel, periodic=(True, True, False),
                       max_coord=24, E=1e3, wall_E=1e3)
        dem.run_substeps(17)
        dem.run_simulation()
        dem.check_status()
        res.append((dem.active_contacts(), dem.gf.position.to_numpy(), dem.gf.omega.to_numpy()))
    monkeypatch.delenv("LBDEM_DEM_KERNELS", raising=False)
    assert set(res[0][0]) == set(res[1][0]) and len(res[0][0]) > 100
    assert np.abs(res[0][1] - res[1][1]).max() < 1e-11
    assert relmax(res[0][2], res[1][2]) < 1e-8


@pytest.mark.parametrize("side", [2, 3])
def test_dem_few_particles_one_block_matches_split_kernels(side, monkeypatch):
    """With at most 64 particles the default single launch is one block
    (block barriers between the phases; 128 threads up to 16 particles, 512
    above): same contact sets and states as two launches per sub-step."""
    rng = np.random.default_rng(14)
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"), -1).reshape(-1, 3)
    pos = 4.5 + g * 3.95 + rng.uniform(-0.05, 0.05, g.shape)
    n = len(pos)
    rad = 2.0 + rng.uniform(-0.02, 0.02, n)
    vel = rng.normal(0, 0.02, (n, 3))
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    res = []
    for m in (None, "split"):
        if m is None:
            monkeypatch.delenv("LBDEM_DEM_KERNELS", raising=False)
        else:
            monkeypatch.setenv("LBDEM_DEM_KERNELS", m)
        dem = make_dem((0.0, 20.0, 0.0, 20.0, 0.0, 16.0), 0.05, (0, 0, -1e-3), _hertz(), rad, mass, pos, vel,
                       periodic=(True, True, False), max_coord=24, E=1e3, wall_E=1e3)
        dem.run_substeps(17)
        dem.check_status()
        res.append((dem.active_contacts(), dem.gf.position.to_numpy(), dem.gf.omega.to_numpy()))
    monkeypatch.delenv("LBDEM_DEM_KERNELS", raising=False)
    assert set(res[0][0]) == set(res[1][0]) and len(res[0][0]) >= (20 if side == 3 else 1)
    assert np.abs(res[0][1] - res[1][1]).max() < 1e-11
    assert relmax(res[0][2], res[1][2]) < 1e-8
