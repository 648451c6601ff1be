"""Map reuse: when no particle's lattice centre or mapping radius changed since
the previous exact map (and the cell types did not change), the owner keys
are already exact and the map only refreshes the particle table and the force
accumulators.  Checked bit for bit against the same lattice with reuse
disabled: a frozen bed, a moving suspension, and a cell-type change between
steps."""
import numpy as np
import pytest

from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu


def _pair_lattices(frozen, seed=3):
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    rng = np.random.default_rng(seed)
    nx, ny, nz = 48, 40, 36
    pos, rad = rsa_spheres(rng, 8, (nx, ny, nz), 6.0, 9.0, gap=1.0, margin=1.0)
    n = len(rad)
    vel = np.zeros((n, 3)) if frozen else rng.normal(0, 2e-3, (n, 3))
    out = []
    for reuse in (True, False):
        dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.2, (0, 0, 0),
                       HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9),
                       rad, 2.0 * 4.0 / 3.0 * np.pi * rad ** 3, pos, vel, periodic=(True, True, True),
                       freeze=np.ones(n, np.int32) if frozen else None)
        lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem, body_force=(2e-5, 0, 0))
        if not reuse:
            lat._psc.map_moved = None
        lat.initialize()
        out.append((lat, dem))
    return out


def _same(a, b, exact_populations=True):
    """Keys bit for bit; forces to FP64 summation order (the per-particle
    reduction adds warp partials atomically, in no fixed order)."""
    (la, da), (lb, db) = a, b
    assert np.array_equal(la._key.cpu().numpy(), lb._key.cpu().numpy())
    np.testing.assert_allclose(da.gf.force_fluid.to_numpy(), db.gf.force_fluid.to_numpy(), rtol=1e-11, atol=1e-20)
    np.testing.assert_allclose(da.gf.moment_fluid.to_numpy(), db.gf.moment_fluid.to_numpy(), rtol=1e-11,
                               atol=1e-20)
    fa, fb = la._f[la._cur].cpu().numpy(), lb._f[lb._cur].cpu().numpy()
    if exact_populations:
        assert np.array_equal(fa, fb)
    else:
        assert np.abs(fa - fb).max() < 1e-9


def test_frozen_bed_reuses_the_map():
    a, b = _pair_lattices(frozen=True)
    for _ in range(6):
        for lat, _ in (a, b):
            lat.step(2)
        _same(a, b)
    # the last call's flag says nothing moved
    lat = a[0]
    assert lat._map_moved.cpu().numpy()[1 - lat._psc.map_parity] == 0


def test_moving_particles_remap():
    a, b = _pair_lattices(frozen=False)
    for _ in range(6):
        for lat, _ in (a, b):
            lat.step(2)
        _same(a, b, exact_populations=False)   # particle velocities carry the force summation order
    lat = a[0]
    assert lat._map_moved.cpu().numpy()[1 - lat._psc.map_parity] == 1


def test_cell_type_change_forces_a_remap():
    from lbdem_taichi_b200.lbm3d.lbmutils import CellType
    a, b = _pair_lattices(frozen=True)
    for lat, _ in (a, b):
        lat.step(1)
        lat.step(1)
    # obstacles through the bed: map-skip cells lose their owner keys
    for lat, _ in (a, b):
        ct = lat.CT.to_numpy()
        ct[20:24, :, :] = CellType.OBSTACLE
        lat.CT.from_numpy(ct)
        lat.step(1)
        lat.step(1)
    _same(a, b)
    key = a[0]._key.cpu().numpy().reshape(36, 40, 48)
    assert not key[:, :, 20:24].any()
