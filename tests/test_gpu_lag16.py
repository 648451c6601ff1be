"""FP32 populations with the lagged Smagorinsky state in FP16
(lagged_storage="f16").

The option stores (drho, u, omega) of each collision as FP16 and reads them
back at the next one, so it must equal the FP32 form whose lagged state is
rounded to FP16 (round to nearest even) after every step -- exactly, for the
populations, the lagged state and the moments, with PSC particles, walls and
open boundaries (boundary pass), and with the row-staged kernel requested
(which leaves this option to the gathering kernel).  Particles are frozen so
both runs map the same positions; forces are compared to 1e-12 relative (the
FP64 force atomics sum in a different order run to run).  Its error against
FP64 at full size is in test_gpu_fullsize.py.
"""
import os

import numpy as np
import pytest
import torch

from tests.gpu_util import make_dem, rsa_spheres

pytestmark = pytest.mark.gpu

FLUID, OBST, INLET, PRE_ZOUHE, LEFT, RIGHT = 1, 8, 262144, 256, 8192, 4096


def _hertz():
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    return HertzContactConfig(pp_friction=0.3, pp_restitution=0.9, pw_friction=0.3, pw_restitution=0.9)


def _run(shape, walls, lag16, round_between, steps=8, kernel=None, seed=3):
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    if kernel:
        os.environ["LBDEM_STEP_KERNEL"] = kernel
    try:
        nx, ny, nz = shape
        rng = np.random.default_rng(seed)
        pos, rad = rsa_spheres(rng, 5, shape, 5.0, 8.0, gap=0.5, margin=1.5)
        vel = rng.normal(0, 2e-3, (5, 3))
        mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
        dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (0, 0, 0), _hertz(), rad, mass, pos, vel,
                       periodic=(walls != "open", True, walls is None), freeze=np.ones(5, np.int32))
        lat = PSCLattice3D(nx, ny, nz, 1 / 0.55, 1.0, 1.0, 1.0, dem, smagorinsky="reference",
                           body_force=(2e-5, 0, 4e-6), storage="f32", lagged_storage="f16" if lag16 else None)
        assert lat._aux.dtype == (torch.float16 if lag16 else torch.float32)
        ct = np.full(shape, FLUID, np.int32)
        if walls is not None:
            ct[:, :, 0] = ct[:, :, -1] = OBST
        if walls == "open":
            ct[0] = INLET | LEFT
            ct[-1] = PRE_ZOUHE | RIGHT
            lat.CT.from_numpy(ct)
            v = np.zeros(shape + (3,))
            v[0, ..., 0] = 0.02
            lat.vel.from_numpy(v)
        elif walls is not None:
            lat.CT.from_numpy(ct)
        lat.initialize()
        if round_between:
            lat._aux.copy_(lat._aux.half().float())
        for _ in range(steps):
            lat.collide()
            lat.stream()
            if round_between:
                lat._aux.copy_(lat._aux.half().float())
        lat.check_status()
        return (lat.f.to_numpy(), lat.rho.to_numpy(), lat.vel.to_numpy(), lat._aux.float().cpu().numpy(),
                dem.gf.force_fluid.to_numpy())
    finally:
        if kernel:
            del os.environ["LBDEM_STEP_KERNEL"]


@pytest.mark.parametrize("shape,walls", [((64, 40, 36), None), ((70, 30, 28), "obstacle"),
                                         ((64, 30, 28), "open")])
def test_lag16_equals_fp32_with_rounded_lagged_state(shape, walls):
    a = _run(shape, walls, lag16=False, round_between=True)
    b = _run(shape, walls, lag16=True, round_between=False)
    for k in range(4):
        np.testing.assert_array_equal(b[k], a[k])
    np.testing.assert_allclose(b[4], a[4], rtol=1e-12, atol=1e-12 * np.abs(a[4]).max())
    assert np.abs(a[4]).max() > 0


def test_lag16_with_row_kernel_requested():
    a = _run((64, 40, 36), None, lag16=True, round_between=False, kernel="simt")
    b = _run((64, 40, 36), None, lag16=True, round_between=False, kernel="rows")
    for k in range(4):
        np.testing.assert_array_equal(b[k], a[k])


def test_lag16_differs_from_fp32_by_the_rounding_only():
    a = _run((64, 40, 36), None, lag16=False, round_between=False)
    b = _run((64, 40, 36), None, lag16=True, round_between=False)
    assert not np.array_equal(a[0], b[0])
    # f - w over eight steps: the FP16 lagged state moves populations by far less than their deviations
    dev = np.abs(a[0] - np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)).max()
    assert np.abs(a[0] - b[0]).max() <= 1e-3 * dev


def test_lagged_storage_arguments():
    from lbdem_taichi_b200.lbm3d.lattice import BasicLattice3D
    for storage, lag in (("f16", "f32"), ("bf16", "f16"), ("f32", "bf16")):
        with pytest.raises(ValueError):
            BasicLattice3D(32, 8, 8, 1.6, 1.0, 1.0, 1.0, smagorinsky="reference", storage=storage, lagged_storage=lag)
    lat = BasicLattice3D(32, 8, 8, 1.6, 1.0, 1.0, 1.0, smagorinsky="reference", storage="f16", lagged_storage="f16")
    assert lat._aux.dtype == torch.float16 and lat.lagged_storage == "f16"
