"""Degenerate and ragged lattice shapes on the GPU against the FP64 oracle:
a lattice narrower than one x-block (Nx = 5), a row of one full and one
one-cell x-block (Nx = 33), and one-cell-thick periodic axes (Ny = 1,
Nz = 1).  Fused step with lagged Smagorinsky, body force and a PSC sphere;
the pipelined run() on the ragged shapes against the sequential loop.

Tolerances as the larger oracle cases: owner ids exact, FP32 populations
absolute 2e-6, particle force / torque max error / max magnitude <= 2e-4;
pipelined vs sequential populations absolute 1e-6 (the force sums that move
the particles are added in another order).
"""
import numpy as np
import pytest

from tests.golden_util import relmax
from tests.test_gpu_oracle import FLUID, _pair

pytestmark = pytest.mark.gpu

SHAPES = [
    # (shape, sphere centre, radius, z walls)
    ((5, 12, 10), (2.3, 5.7, 4.9), 2.6, True),
    ((33, 10, 12), (16.2, 4.6, 5.8), 3.7, True),
    ((40, 1, 24), (19.7, 0.4, 11.3), 4.2, True),
    ((24, 16, 1), (11.6, 7.7, 0.45), 4.1, False),
]


@pytest.mark.parametrize("shape,centre,radius,walls", SHAPES)
def test_shapes_vs_oracle(shape, centre, radius, walls):
    rng = np.random.default_rng(31)
    nx, ny, nz = shape
    pos = np.array([centre], float)
    rad = np.array([radius])
    vel = np.array([[1.5e-3, -1e-3, 5e-4]])
    omg = np.array([[1e-3, 2e-3, -1e-3]])
    ct = None if walls else np.full(shape, FLUID, np.int32)
    periodic = (True, True, not walls)
    lat, dem, o, od, og = _pair(nx, ny, nz, pos, rad, vel, omg, force=(2e-6, -1e-6, 0.0), ct=ct,
                                periodic=periodic)
    u0 = 0.02 * rng.uniform(-1, 1, (nx, ny, nz, 3))
    r0 = 1.0 + 0.002 * rng.uniform(-1, 1, (nx, ny, nz))
    lat.vel.from_numpy(u0)
    lat.rho.from_numpy(r0)
    o.vel[...] = u0
    o.rho[...] = r0
    lat.initialize()
    o.initialize()
    fl = o.ct == FLUID
    for s in range(6):
        lat.collide()
        o.grains2lattice(og)
        o.collide()
        o.lattice2grains(og)
        np.testing.assert_array_equal(lat.id.to_numpy(), o.id)
        assert relmax(dem.gf.force_fluid.to_numpy(), og.force_fluid) < 2e-4, s
        assert relmax(dem.gf.moment_fluid.to_numpy(), og.moment_fluid) < 2e-4, s
        lat.stream()
        o.stream()
    assert (o.id >= 0).any()
    assert np.abs(lat.f.to_numpy() - o.f)[fl].max() < 2e-6
    assert relmax(lat.vel.to_numpy()[fl], o.vel[fl]) < 1e-4
    lat.check_status()


@pytest.mark.parametrize("shape,centre,radius,walls", SHAPES[:3])
def test_shapes_pipelined_run(shape, centre, radius, walls):
    nx, ny, nz = shape
    out = []
    for pipeline in (False, True):
        lat, dem, *_ = _pair(nx, ny, nz, np.array([centre], float), np.array([radius]),
                             np.array([[2e-3, 1e-3, -5e-4]]), None, force=(2e-6, 0.0, 0.0))
        lat.initialize()
        lat.run(34, 5, pipeline=pipeline)
        lat.check_status()
        dem.check_status()
        out.append((lat.f.to_numpy(), dem.gf.position.to_numpy()))
    (f0, p0), (f1, p1) = out
    assert np.abs(f0 - f1).max() < 1e-6
    assert np.abs(p0 - p1).max() < 1e-9
