"""Periodic images (DEMSolver(..., compat="wrapped")): the PSC map, the
coupled forces and the DEM broad phase see a sphere or a contact pair that
crosses a periodic face exactly as the same configuration shifted by a whole
number of cells into the interior.  The reference mode drops the part beyond
the face (no images in grains2lattice, psclattice3d.py:102-108; no pairs across
periodic faces in the broad phase, bpcd.py:154-194), which the tests show too.

Tolerances: owner ids and solid fractions exact; particle force and torque
max error / max magnitude <= 1e-5 (FP32 lattice, different summation order);
DEM velocities (FP64) 1e-9 relative and positions 1e-9 absolute to the shifted run.
"""
import numpy as np
import pytest

from tests.gpu_util import make_dem

pytestmark = pytest.mark.gpu

NX, NY, NZ = 48, 40, 36


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)


def _lattice(centres, compat, rad=6.0):
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    pos = np.asarray(centres, float)
    n = len(pos)
    radius = np.full(n, rad)
    vel = np.tile([2e-3, -1e-3, 5e-4], (n, 1))
    omg = np.tile([1e-3, 2e-3, -1e-3], (n, 1))
    dem = make_dem((0.0, NX, 0.0, NY, 0.0, NZ), 0.1, (0, 0, 0), _hertz(), radius, 2.0 * 4 / 3 * np.pi * radius ** 3,
                   pos, vel, omega=omg, periodic=(True, True, True), compat=compat)
    lat = PSCLattice3D(NX, NY, NZ, 1 / 0.6, 1.0, 1.0, 1.0, dem, body_force=(1e-5, 0.0, 0.0))
    v = np.zeros((NX, NY, NZ, 3))
    v[..., 0], v[..., 1] = 0.01, 0.004
    lat.vel.from_numpy(v)
    return lat, dem


# lattice centre (xc) = position + 0.5 (psclattice3d.py:102); the first sphere crosses the x = 0 face,
# the second the y and z faces (a corner image).  Centres off the 0.1 grid: with centres on it many of
# the 0.2-spaced sub-points lie exactly on the sphere surface, where FP64 rounding (here and in the
# reference alike) decides differently for differently translated copies.
STRADDLE = [[1.73412, 20.31753, 17.61291], [24.21937, 38.91372, 0.81234]]
SHIFT = (12, 10, 8)   # moves both spheres at least one reach inside every face


def _shifted(c):
    return [[(p[0] + SHIFT[0]) % NX, (p[1] + SHIFT[1]) % NY, (p[2] + SHIFT[2]) % NZ] for p in c]


def _roll(a):
    # a[x, y, z, ...] of the shifted run, moved back onto the straddling run's cells
    return np.roll(a, shift=(-SHIFT[0], -SHIFT[1], -SHIFT[2]), axis=(0, 1, 2))


def test_map_with_periodic_images_is_translation_invariant():
    lat_w, _ = _lattice(STRADDLE, "wrapped")
    lat_s, _ = _lattice(_shifted(STRADDLE), "wrapped")
    lat_r, _ = _lattice(STRADDLE, "reference")
    for lat in (lat_w, lat_s, lat_r):
        lat.initialize()
    vf_w, vf_s, vf_r = lat_w.volfrac.to_numpy(), lat_s.volfrac.to_numpy(), lat_r.volfrac.to_numpy()
    np.testing.assert_array_equal(vf_w, _roll(vf_s))
    np.testing.assert_array_equal(lat_w.id.to_numpy(), _roll(lat_s.id.to_numpy()))
    # the reference mode loses the cells beyond the faces; images restore them
    assert vf_r.sum() < vf_w.sum() - 50
    assert abs(vf_w.sum() - vf_s.sum()) < 1e-9


def test_coupled_forces_with_periodic_images_are_translation_invariant():
    runs = {}
    for key, cen, compat in (("w", STRADDLE, "wrapped"), ("s", _shifted(STRADDLE), "wrapped"),
                             ("r", STRADDLE, "reference")):
        lat, dem = _lattice(cen, compat)
        lat.initialize()
        for _ in range(5):
            lat.collide()
            lat.stream()
        runs[key] = (dem.gf.force_fluid.to_numpy(), dem.gf.moment_fluid.to_numpy(), lat)
        lat.check_status()
    Fw, Mw, lw = runs["w"]
    Fs, Ms, ls = runs["s"]
    Fr, _, _ = runs["r"]
    assert np.abs(Fw - Fs).max() <= 1e-5 * np.abs(Fs).max(), (Fw, Fs)
    assert np.abs(Mw - Ms).max() <= 1e-5 * np.abs(Ms).max(), (Mw, Ms)
    np.testing.assert_allclose(lw.rho.to_numpy(), _roll(ls.rho.to_numpy()), rtol=0, atol=2e-6)
    # without images the straddling spheres feel a different (truncated) force
    assert np.abs(Fr - Fs).max() > 0.05 * np.abs(Fs).max()


def _dem_pair(x0, compat, L=120.0):
    """Two d = 12 spheres approaching each other along x; the pair straddles
    the x faces when x0 is near 0."""
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    r = 6.0
    pos = np.array([[x0 - 5.9, 60.0, 60.0], [x0 + 5.9, 61.0, 59.5]])
    pos[:, 0] %= L
    vel = np.array([[1e-3, 0.0, 0.0], [-1e-3, 2e-4, 0.0]])
    return make_dem((0.0, L, 0.0, L, 0.0, L), 0.05, (0, 0, 0),
                    HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9),
                    np.full(2, r), np.full(2, 2.0 * 4 / 3 * np.pi * r ** 3), pos, vel,
                    periodic=(True, True, True), compat=compat)


def test_dem_contacts_across_periodic_faces():
    a = _dem_pair(0.3, "wrapped")     # straddles x = 0
    b = _dem_pair(40.3, "wrapped")    # same pair, interior
    c = _dem_pair(0.3, "reference")   # straddles, no images: never collides
    for d in (a, b, c):
        d.run_substeps(40)
    va, vb, vc = (d.gf.velocity.to_numpy() for d in (a, b, c))
    np.testing.assert_allclose(va, vb, rtol=1e-9, atol=1e-15)
    pa = a.gf.position.to_numpy()
    pb = b.gf.position.to_numpy()
    dx = (pa - pb + np.array([40.0, 0, 0])) % 120.0
    dx[dx > 60.0] -= 120.0
    assert np.abs(dx).max() < 1e-9
    # the contact changed the velocities; without images nothing happened
    assert np.abs(vb - np.array([[1e-3, 0, 0], [-1e-3, 2e-4, 0]])).max() > 1e-4
    np.testing.assert_allclose(vc, [[1e-3, 0, 0], [-1e-3, 2e-4, 0]], rtol=0, atol=1e-15)
    for d in (a, b, c):
        d.check_status()


def test_short_periodic_length_is_refused():
    from lbdem_taichi_b200._native import LbdemError
    d = _dem_pair(10.0, "wrapped", L=80.0)   # 80 < 4 broad-phase cells of 24
    with pytest.raises(LbdemError, match="periodic length"):
        d.run_substeps(1)
