"""Pipelined run(): the x-blocks no particle can reach are stepped while the
DEM and the next map run on a second stream, the near blocks after the map.
Compared with the sequential loop (collide, stream, DEM) on identical
lattices.

Tolerances: populations max |diff| <= 1e-6 (FP32) / 1e-5 in storage units of
the 16-bit forms (both runs take the same FP32 path; the only difference is
the order of the FP64 atomic force sums, which moves the particles by
~1e-16); particle forces 1e-9 relative; positions 1e-9 absolute.
"""
import numpy as np
import pytest

from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)


def _suspension(storage="f32", seed=5, n=40, shape=(96, 80, 72)):
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    pos, rad = rsa_spheres(rng, n, shape, 8.0, 12.0, gap=1.0, margin=0.5)
    vel = rng.normal(0, 2e-3, (len(rad), 3))
    dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (1e-6, 0, 0), _hertz(), rad,
                   2.0 * 4 / 3 * np.pi * rad ** 3, pos, vel, periodic=(True, True, True))
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem, smagorinsky="reference",
                       body_force=(1e-6, 0, 0), storage=storage)
    lat.initialize()
    return lat, dem


def _compare(a, b, ftol):
    (la, da), (lb, db) = a, b
    fa = la._f[la._cur].float().cpu().numpy()
    fb = lb._f[lb._cur].float().cpu().numpy()
    assert la._cur == lb._cur and la._cur_kind == lb._cur_kind
    assert np.abs(fa - fb).max() <= ftol, np.abs(fa - fb).max()
    Fa, Fb = da.gf.force_fluid.to_numpy(), db.gf.force_fluid.to_numpy()
    assert np.abs(Fa - Fb).max() <= 1e-9 * np.abs(Fb).max()
    assert np.abs(da.gf.position.to_numpy() - db.gf.position.to_numpy()).max() <= 1e-9
    assert np.array_equal(la._key.cpu().numpy(), lb._key.cpu().numpy())


@pytest.mark.parametrize("storage,ftol", [("f32", 1e-6), ("f16", 1e-5 * 4096)])
def test_pipelined_run_equals_sequential_loop(storage, ftol):
    a = _suspension(storage)
    b = _suspension(storage)
    a[0].run(12, 10, pipeline=True)
    for _ in range(12):
        b[0].step(10)
    _compare(a, b, ftol)
    for lat, dem in (a, b):
        lat.check_status()
        dem.check_status()
    # the particles moved and the near blocks are a small part of the lattice
    near = a[0]._near.cpu().numpy()
    assert 0 < near.mean() < 0.6


def test_pipelined_run_with_open_boundaries():
    """Packed bed between a Ladd inlet and a Zou-He pressure outlet: the
    boundary pass follows the near-block phase."""
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    nx, ny, nz = 80, 40, 36
    out = []
    for _ in range(2):
        rng = np.random.default_rng(9)
        pos, rad = rsa_spheres(rng, 10, (nx - 30, ny, nz), 7.0, 9.0, gap=1.0, margin=1.0)
        pos[:, 0] += 15.0
        n = len(rad)
        dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (0, 0, 0), _hertz(), rad, 2.0 * 4 / 3 * np.pi * rad ** 3,
                       pos, np.zeros((n, 3)), periodic=(False, True, True), freeze=np.ones(n, np.int32))
        lat = PSCLattice3D(nx, ny, nz, 1 / 0.68, 1.0, 1.0, 1.0, dem)
        ct = np.ones((nx, ny, nz), np.int32)
        ct[0] = 262144 | 8192      # VEL_INLET_LADD | LEFT
        ct[-1] = 256 | 4096        # Pre_ZOUHE | RIGHT
        lat.CT.from_numpy(ct)
        v = np.zeros((nx, ny, nz, 3))
        v[0, :, :, 0] = 0.01
        lat.vel.from_numpy(v)
        lat.initialize()
        out.append((lat, dem))
    out[0][0].run(15, 1, pipeline=True)
    for _ in range(15):
        out[1][0].step(1)
    _compare(out[0], out[1], 1e-6)
    np.testing.assert_allclose(out[0][0].rho.to_numpy(), out[1][0].rho.to_numpy(), rtol=0, atol=1e-6)
    out[0][0].check_status()


def test_particle_beyond_the_margin_is_flagged():
    """A particle that moves more than the pipeline margin in one step is
    reported (its new cells may have been stepped as plain fluid)."""
    from lbdem_taichi_b200 import _native as N
    lat, dem = _suspension(n=6, seed=8, shape=(64, 64, 64))
    vel = dem.gf.velocity.to_numpy()
    vel[0] = (2.0, 0.0, 0.0)            # DEM dt 0.1: 0.2 lattice units per sub-step, 2 per step
    dem.gf.velocity.from_numpy(vel)
    lat.pipeline_margin = 1.0
    lat.run(3, 10, pipeline=True)
    assert int(lat._status.item()) & N.ST_PIPELINE_MARGIN
    lat.clear_status()


@pytest.mark.parametrize("storage,ftol", [("f32", 1e-6), ("f16", 1e-5 * 4096)])
def test_sequential_run_with_early_key_clear(storage, ftol):
    """run(pipeline=False) clears each map's keys beside the DEM
    (lbdem_psc_map_clear) rather than in the next map: the same as step() n
    times, and the last map's keys stay for the fields read after it."""
    a = _suspension(storage)
    b = _suspension(storage)
    a[0].run(12, 10, pipeline=False)
    for _ in range(12):
        b[0].step(10)
    _compare(a, b, ftol)
    assert a[0]._psc.have_prev == 1
    np.testing.assert_array_equal(a[0].volfrac.to_numpy(), b[0].volfrac.to_numpy())
    assert a[0].volfrac.to_numpy().max() == 1.0
    for lat, dem in (a, b):
        lat.check_status()
        dem.check_status()
