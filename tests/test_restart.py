"""Population and particle checkpoint/restart (the reference has none: its
drivers pickle macroscopic snapshots only).  A run continued from a saved
state matches the uninterrupted run: populations bit for bit (same kernels on
the same inputs), particle state to FP64 rounding (the order of the atomic
force sums differs)."""
import numpy as np
import pytest

from tests.golden_util import relmax
from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu


def _build(storage, smag):
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    rng = np.random.default_rng(5)
    nx, ny, nz = 40, 32, 24
    pos, rad = rsa_spheres(rng, 8, (nx, ny, nz), 5.0, 7.0, gap=0.3, margin=1.0)
    vel = rng.normal(0, 2e-3, (8, 3))
    mass = 2.0 * 4 / 3 * np.pi * rad ** 3
    dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (0, 0, -2e-5),
                   HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9),
                   rad, mass, pos, vel, periodic=(True, True, False), E=1e3, wall_E=1e3)
    lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem, smagorinsky=smag, body_force=(1e-5, 0, 0),
                       storage=storage)
    ct = np.full((nx, ny, nz), 1, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = 8
    lat.CT.from_numpy(ct)
    lat.initialize()
    return lat, dem


@pytest.mark.parametrize("storage,smag", [("f32", "reference"), ("f16", "off")])
def test_restart_continues_the_run(tmp_path, storage, smag):
    lat, dem = _build(storage, smag)
    lat.run(6, sub_cycles=10)
    lat.save_state(tmp_path / "lat.pt")
    dem.save_state(tmp_path / "dem.pt")
    lat.run(5, sub_cycles=10)
    fa, pa, ffa = lat.f.to_numpy(), dem.gf.position.to_numpy(), dem.gf.force_fluid.to_numpy()
    lat.check_status()

    lat2, dem2 = _build(storage, smag)
    lat2.load_state(tmp_path / "lat.pt")
    dem2.load_state(tmp_path / "dem.pt")
    lat2.run(5, sub_cycles=10)
    fb, pb, ffb = lat2.f.to_numpy(), dem2.gf.position.to_numpy(), dem2.gf.force_fluid.to_numpy()
    assert np.array_equal(fa, fb)
    assert np.abs(pa - pb).max() < 1e-12
    assert relmax(ffa, ffb) < 1e-9
    assert len(dem2.active_contacts()) == len(dem.active_contacts())
