"""Gradients of the drag on a frozen particle bed: hand-written reverse mode of
the fused PSC step, behind a ``torch.autograd.Function``.

The reference has no gradients.  This module differentiates exactly what
``PSCLattice3D.collide(); stream()`` computes for N steps
(psclattice3d.py:187-358, lbm_solver3d.py:197-240, lbm_foecelover.py:52-68)
on a bed of frozen particles, with respect to the uniform body force and the
particle centres, for the loss

    L = e . sum_particles force_fluid   (after the N-th collide)

i.e. the total hydrodynamic force on the bed along e at step N.  Particle
positions enter the step only through the solid fraction, which must be the
lattice's ``solid_fraction="smooth"`` map (the reference's 5^3 count is
piecewise constant in the positions).

Memory: the forward run keeps the populations every ``checkpoint_every``
steps; the backward run recomputes one segment of states from its checkpoint
and runs the adjoint steps (lbdem_psc_step_adjoint_f32) back through it.

    lat = PSCLattice3D(nx, ny, nz, omega, dx, dt, rho, dem, body_force=(gx, 0, 0),
                       solid_fraction="smooth")
    prob = FrozenBedDrag(lat, n_steps=500, direction=(1, 0, 0), checkpoint_every=50)
    F = torch.tensor([gx, 0, 0], dtype=torch.float64, requires_grad=True)
    P = torch.tensor(positions, dtype=torch.float64, requires_grad=True)
    loss = drag_loss(F, P, prob)
    loss.backward()          # F.grad, P.grad
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _native as N
from .psclattice3d import PSCLattice3D


class FrozenBedDrag:
    """Forward run with checkpoints and its reverse sweep for one lattice."""

    def __init__(self, lattice: PSCLattice3D, n_steps: int, direction=(1.0, 0.0, 0.0), checkpoint_every: int = 50):
        lat = lattice
        if lat.solid_fraction != "smooth":
            raise ValueError('the drag gradient needs PSCLattice3D(..., solid_fraction="smooth")')
        if lat.storage != "f32" or lat.smagorinsky != "off":
            raise ValueError("the adjoint covers FP32 storage with Smagorinsky off")
        if lat.dem.n == 0:
            raise ValueError("no particles")
        lat._sync_inputs()
        if lat.has_moving_walls or lat.has_open_boundaries:
            raise ValueError("the adjoint covers fixed walls (OBSTACLE) only, not moving walls (VEL_LADD), "
                             "inlets or other open boundaries")
        if int(n_steps) < 1 or int(checkpoint_every) < 1:
            raise ValueError("n_steps and checkpoint_every must be positive")
        self.lat = lat
        self.n_steps = int(n_steps)
        self.K = int(checkpoint_every)
        self.direction = np.asarray(direction, np.float64).reshape(3)
        self._dir = torch.tensor(self.direction, dtype=torch.float64, device="cuda")
        self._ckpt = {}
        self.loss = None

    # ------------------------------------------------------------ parameters
    def set_parameters(self, force=None, positions=None):
        """Body force (3, lattice units) and particle centres ((n, 3), physical)."""
        lat = self.lat
        if force is not None:
            f = np.asarray(force, np.float64).reshape(3)
            lat.body_force = f
            lat._fill_desc()
        if positions is not None:
            p = torch.as_tensor(positions, dtype=torch.float64).reshape(lat.dem.n, 3)
            lat.dem._t["position"].copy_(p.to(lat.dem._t["position"].device))
            lat.dem._touched("position")

    # ------------------------------------------------------------ forward
    def forward(self) -> float:
        """Initialize and run n_steps; returns L and keeps the checkpoints."""
        lat = self.lat
        lat.initialize()
        self._ckpt = {0: lat._f[lat._cur].clone()}
        for n in range(1, self.n_steps + 1):
            lat.collide()
            lat.stream()
            if n % self.K == 0 and n < self.n_steps:
                self._ckpt[n] = lat._f[lat._cur].clone()
        ff = lat.dem._t["force_fluid"]
        self.loss = float((ff.sum(dim=0) * self._dir).sum().item())
        return self.loss

    # ------------------------------------------------------------ reverse
    def _step(self, Ld, src, dst, gather):
        """One forward step kernel from buffer src into dst (recompute)."""
        Ld.f[0], Ld.f[1] = N.ptr(src), N.ptr(dst)
        N.call("lbdem_psc_step_f32", C.byref(Ld), C.byref(self.lat._psc), C.byref(self.lat._grains), 0, 1,
               int(gather), N.stream_handle())

    def backward(self):
        """Returns (dL/dF (3,) in lattice units, dL/dpos (n, 3) physical)."""
        if self.loss is None:
            raise RuntimeError("run forward() first")
        lat = self.lat
        lat._sync_inputs()
        Ld = N.Lattice.from_buffer_copy(lat._lat)   # same lattice, buffers repointed per call
        like = lat._f[0]
        lam = [torch.zeros_like(like), torch.zeros_like(like)]
        bbar = torch.zeros(lat.ncells, dtype=torch.float32, device="cuda")
        gbar = torch.zeros(3, dtype=torch.float64, device="cuda")
        dirv = (C.c_double * 3)(*self.direction)
        states = [torch.empty_like(like) for _ in range(self.K)]
        cur = 0
        N_ = self.n_steps
        seg_starts = list(range(0, N_, self.K))
        for s0 in reversed(seg_starts):
            s1 = min(s0 + self.K, N_)
            # states[i] = populations read by step s0 + 1 + i
            states[0].copy_(self._ckpt[s0])
            for i in range(1, s1 - s0):
                self._step(Ld, states[i - 1], states[i], gather=(s0 + i) >= 2)
            for n in range(s1, s0, -1):
                i = n - 1 - s0
                seed = n == N_
                gather = n >= 2
                N.call("lbdem_psc_step_adjoint_f32", C.byref(Ld), C.byref(lat._psc), N.ptr(states[i]),
                       None if seed else N.ptr(lam[cur]), N.ptr(lam[1 - cur]), N.ptr(bbar), N.ptr(gbar), dirv,
                       int(gather), int(seed), N.stream_handle())
                cur = 1 - cur
        pos_bar = torch.zeros((lat.dem.n, 3), dtype=torch.float64, device="cuda")
        N.call("lbdem_psc_force_adjoint", C.byref(Ld), C.byref(lat._psc), C.byref(lat._grains), N.ptr(bbar),
               N.ptr(pos_bar), N.stream_handle())
        lat.check_status()
        self.bbar = bbar
        return gbar.cpu().numpy(), pos_bar.cpu().numpy()


class _DragFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, force, positions, problem):
        problem.set_parameters(force.detach().cpu().numpy(), positions.detach())
        loss = problem.forward()
        ctx.problem = problem
        ctx.devs = (force.device, positions.device)
        return torch.tensor(loss, dtype=torch.float64, device=force.device)

    @staticmethod
    def backward(ctx, gout):
        gF, gP = ctx.problem.backward()
        g = float(gout.item())
        return (torch.as_tensor(gF * g, device=ctx.devs[0]), torch.as_tensor(gP * g, device=ctx.devs[1]), None)


def drag_loss(force: torch.Tensor, positions: torch.Tensor, problem: FrozenBedDrag) -> torch.Tensor:
    """Differentiable L(force, positions) for ``problem`` (see module doc)."""
    return _DragFn.apply(force, positions, problem)
