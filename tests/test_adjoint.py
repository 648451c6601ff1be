"""Reverse mode of the PSC step on a frozen bed (drag gradients).

Loss: L = e . sum_particles force_fluid after N steps of the channel flow
driven by a body force F, with the smooth solid fraction.  The FP64 oracle's
adjoint (oracle/lbdem_oracle.c, orc_adjoint_*) is pinned to FP64 central
finite differences of the oracle's forward (the reference's collide / stream /
lattice2grains restated); the CUDA adjoint (FP32) is compared with it.

Tolerances: FD vs FP64 adjoint 1e-4 relative (FD truncation of the C1 ramp
dominates for the positions); CUDA FP32 adjoint vs FP64 adjoint 1e-4
relative for dL/dF and 1e-4 of max |dL/dpos| for the positions.
"""
import numpy as np
import pytest

from oracle.oracle import frozen_bed_drag

from tests.gpu_util import rsa_spheres

FLUID, OBST = 1, 8
OMEGA = 1 / 0.6


def _channel(nx, ny, nz):
    ct = np.full((nx, ny, nz), FLUID, np.int32)
    ct[:, :, 0] = ct[:, :, -1] = OBST
    return ct


def _bed(seed, box, n, dmin, dmax):
    rng = np.random.default_rng(seed)
    pos, rad = rsa_spheres(rng, n, box, dmin, dmax, gap=1.5, margin=1.5)
    assert len(rad) == n
    return pos, rad


def test_oracle_adjoint_matches_central_differences():
    nx, ny, nz = 16, 12, 14
    ct = _channel(nx, ny, nz)
    pos = np.array([[5.3, 6.1, 4.7], [11.2, 5.4, 8.9]])
    rad = np.array([2.6, 2.2])
    F = np.array([2e-5, 0.0, 0.0])
    steps = 12
    L, gF, gP = frozen_bed_drag((nx, ny, nz), OMEGA, ct, rad, pos, F, steps, grad=True)
    assert L > 0
    h = 1e-4 * F[0]
    fd = (frozen_bed_drag((nx, ny, nz), OMEGA, ct, rad, pos, F + [h, 0, 0], steps)
          - frozen_bed_drag((nx, ny, nz), OMEGA, ct, rad, pos, F - [h, 0, 0], steps)) / (2 * h)
    assert abs(fd - gF[0]) <= 1e-6 * abs(gF[0])
    big = np.argwhere(np.abs(gP) > 0.05 * np.abs(gP).max())
    assert len(big) >= 3
    for i, k in big:
        hp = 1e-4 * abs(pos[i, k])
        pp, pm = pos.copy(), pos.copy()
        pp[i, k] += hp
        pm[i, k] -= hp
        fdp = (frozen_bed_drag((nx, ny, nz), OMEGA, ct, rad, pp, F, steps)
               - frozen_bed_drag((nx, ny, nz), OMEGA, ct, rad, pm, F, steps)) / (2 * hp)
        assert abs(fdp - gP[i, k]) <= 1e-4 * abs(gP[i, k]), (i, k, fdp, gP[i, k])


def _gpu_problem(nx, ny, nz, pos, rad, F, steps, every, direction=(1.0, 0.0, 0.0)):
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from lbdem_taichi_b200.lbdem.adjoint import FrozenBedDrag
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D

    from tests.gpu_util import make_dem
    n = len(rad)
    mass = 2.0 * 4.0 / 3.0 * np.pi * rad ** 3
    dem = make_dem((0.0, nx, 0.0, ny, 0.0, nz), 0.1, (0, 0, 0),
                   HertzContactConfig(pp_friction=0.3, pw_friction=0.3, pp_restitution=0.9, pw_restitution=0.9),
                   rad, mass, pos, np.zeros((n, 3)), periodic=(True, True, False), freeze=np.ones(n, np.int32))
    lat = PSCLattice3D(nx, ny, nz, OMEGA, 1.0, 1.0, 1.0, dem, body_force=F, solid_fraction="smooth")
    lat.CT.from_numpy(_channel(nx, ny, nz))
    return FrozenBedDrag(lat, steps, direction=direction, checkpoint_every=every)


@pytest.mark.gpu
def test_gpu_adjoint_matches_fp64_adjoint():
    nx, ny, nz = 40, 32, 24
    pos, rad = _bed(5, (nx, ny, nz), 6, 6.0, 9.0)
    F = np.array([2e-6, 0.0, 0.0])
    steps = 40
    Lo, gFo, gPo = frozen_bed_drag((nx, ny, nz), OMEGA, _channel(nx, ny, nz), rad, pos, F, steps, grad=True)
    prob = _gpu_problem(nx, ny, nz, pos, rad, F, steps, every=7)
    L = prob.forward()
    gF, gP = prob.backward()
    assert abs(L - Lo) <= 2e-5 * abs(Lo), (L, Lo)
    assert abs(gF[0] - gFo[0]) <= 1e-4 * abs(gFo[0]), (gF, gFo)
    scale = np.abs(gPo).max()
    assert scale > 0
    assert np.abs(gP - gPo).max() <= 1e-4 * scale, np.abs(gP - gPo).max() / scale


@pytest.mark.gpu
def test_gpu_checkpointing_changes_nothing():
    """Segments of 3 steps recomputed from checkpoints give the gradient of the
    single-segment sweep (same kernels, same states; only the order of the
    FP64 atomic sums may differ)."""
    nx, ny, nz = 32, 24, 20
    pos, rad = _bed(6, (nx, ny, nz), 4, 5.0, 8.0)
    F = np.array([3e-6, 0.0, 1e-7])
    res = []
    for every in (3, 20):
        prob = _gpu_problem(nx, ny, nz, pos, rad, F, 20, every=every, direction=(1.0, 0.5, 0.0))
        L = prob.forward()
        gF, gP = prob.backward()
        res.append((L, gF, gP))
    assert abs(res[0][0] - res[1][0]) <= 1e-12 * abs(res[1][0])
    np.testing.assert_allclose(res[0][1], res[1][1], rtol=1e-12, atol=1e-14 * np.abs(res[1][1]).max())
    np.testing.assert_allclose(res[0][2], res[1][2], rtol=1e-12, atol=1e-12 * np.abs(res[1][2]).max())


@pytest.mark.gpu
def test_drag_loss_autograd_function():
    import torch

    from lbdem_taichi_b200.lbdem.adjoint import drag_loss
    nx, ny, nz = 32, 24, 20
    pos, rad = _bed(7, (nx, ny, nz), 3, 5.0, 8.0)
    F0 = np.array([2e-6, 0.0, 0.0])
    prob = _gpu_problem(nx, ny, nz, pos, rad, F0, 15, every=5)
    F = torch.tensor(F0, dtype=torch.float64, requires_grad=True)
    P = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    loss = drag_loss(F, P, prob)
    (3.0 * loss).backward()
    gF, gP = prob.backward()
    np.testing.assert_allclose(F.grad.numpy(), 3.0 * gF, rtol=1e-12)
    np.testing.assert_allclose(P.grad.numpy(), 3.0 * gP, rtol=1e-12, atol=1e-18)
    Lo = frozen_bed_drag((nx, ny, nz), OMEGA, _channel(nx, ny, nz), rad, pos, F0, 15)
    assert abs(loss.item() - Lo) <= 2e-5 * abs(Lo)
