"""The row-staged steps (rows copied into shared memory by the TMA; one cell
per thread, LBDEM_STEP_KERNEL=rows, or two x-adjacent cells per thread for
16-bit storage and even Nx, =rows2) against the step that gathers with
per-thread loads (=simt): the same arithmetic on the same inputs, so the
populations, the lagged Smagorinsky state and the moments must agree exactly
-- over several steps, for every storage form, with PSC particles, bounce-back
and moving walls (the two-cell kernel runs the one-cell code in warps that
touch them), open boundaries (boundary pass), periodic images, row widths that
are not a multiple of 32 or of 4 (the key and link rows then come by plain
loads; an odd width or an odd number of x-blocks falls back to one cell per
thread) and one-block rows.

The particles are frozen so that both runs map the same positions (the force
sums use FP64 atomics, whose order differs run to run; the DEM would carry that
last-bit noise into the positions).  Forces are compared to 1e-12 relative
for the one-cell kernels for that reason; the two-cell kernel sums each
thread's two cells before the warp reduction, a different FP32 grouping, and
is held to 1e-5 of the largest force.
"""
import os

import numpy as np
import pytest

from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu

FLUID, OBST, VEL_LADD, INLET, PRE_ZOUHE, LEFT, RIGHT = 1, 8, 32, 262144, 256, 8192, 4096


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9)


def _run(kernel, shape, storage, smag, walls, nsp, steps, wrapped=False, seed=5):
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    os.environ["LBDEM_STEP_KERNEL"] = kernel
    try:
        nx, ny, nz = shape
        rng = np.random.default_rng(seed)
        pos, rad = rsa_spheres(rng, nsp, shape, 5.0, 8.0, gap=0.5, margin=0.0 if wrapped else 1.5)
        vel = rng.normal(0, 2e-3, (nsp, 3))
        mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
        periodic = (walls != "open", True, walls is None)
        dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (0, 0, 0), _hertz(), rad, mass, pos, vel,
                       periodic=periodic, freeze=np.ones(nsp, np.int32),
                       compat="wrapped" if wrapped else "reference")
        lat = PSCLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, dem, smagorinsky=smag, body_force=(1e-5, 0, 2e-6),
                           storage=storage)
        ct = np.full(shape, FLUID, np.int32)
        if walls == "obstacle":
            ct[:, :, 0] = ct[:, :, -1] = OBST
        elif walls == "moving":
            ct[:, :, 0] = ct[:, :, -1] = VEL_LADD
        elif walls == "open":
            ct[:, :, 0] = ct[:, :, -1] = OBST
            ct[0] = INLET | LEFT
            ct[-1] = PRE_ZOUHE | RIGHT
        if walls is not None:
            lat.CT.from_numpy(ct)
        if walls in ("moving", "open"):
            v = np.zeros(shape + (3,))
            if walls == "moving":
                v[:, :, 0, 0], v[:, :, -1, 0] = -0.02, 0.02
            else:
                v[0, ..., 0] = 0.01
            lat.vel.from_numpy(v)
        lat.initialize()
        for _ in range(steps):
            lat.collide()
            lat.stream()
        lat.check_status()
        F = dem.gf.force_fluid.to_numpy()
        aux = lat._aux.float().cpu().numpy() if lat._aux is not None else None
        return lat.f.to_numpy(), lat.rho.to_numpy(), lat.vel.to_numpy(), aux, F
    finally:
        del os.environ["LBDEM_STEP_KERNEL"]


CASES = [
    # shape, storage, smagorinsky, walls, spheres, wrapped
    ((64, 48, 40), "f32", "reference", None, 6, False),
    ((64, 48, 40), "f16", "reference", None, 6, False),
    ((64, 48, 40), "bf16", "local", "obstacle", 6, False),
    ((256, 24, 20), "f16", "reference", "obstacle", 8, False),
    ((96, 40, 36), "f32", "off", "moving", 5, False),
    ((70, 30, 28), "f16", "reference", "open", 4, False),     # boundary pass; Nx % 4 = 2: plain key / link loads
    ((45, 33, 31), "f32", "reference", None, 3, False),       # partial last x-block, odd widths
    ((20, 16, 18), "f16", "off", "obstacle", 2, False),       # one x-block
    ((64, 48, 40), "f32", "reference", None, 6, True),        # periodic images
    ((128, 24, 20), "f16", "reference", "open", 4, False),    # two cells per thread beside open boundaries
    ((128, 20, 18), "bf16", "off", "moving", 3, False),       # ... and beside moving walls
    ((64, 40, 36), "f16", "reference", None, 5, True),        # ... with periodic images
]


@pytest.mark.parametrize("kernel", ["rows", "rows2"])
@pytest.mark.parametrize("shape,storage,smag,walls,nsp,wrapped", CASES)
def test_rows_kernel_equals_gather_kernel(kernel, shape, storage, smag, walls, nsp, wrapped):
    a = _run("simt", shape, storage, smag, walls, nsp, 6, wrapped)
    b = _run(kernel, shape, storage, smag, walls, nsp, 6, wrapped)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[1], a[1])
    np.testing.assert_array_equal(b[2], a[2])
    if a[3] is not None:
        np.testing.assert_array_equal(b[3], a[3])
    tol = 1e-5 if kernel == "rows2" else 1e-12
    np.testing.assert_allclose(b[4], a[4], rtol=tol, atol=tol * np.abs(a[4]).max())
    assert np.abs(a[4]).max() > 0
