"""Partially saturated cell (Noble-Torczynski) LBM-DEM coupling on the GPU
(API of src/lbdem/psclattice3d.py:22-358).

``PSCLattice3D(Nx, Ny, Nz, omega, dx, dt, rho, demslover)`` keeps the
reference's constructor and ``initialize / collide / stream`` methods.  Each
``collide()`` maps the DEM particles onto the lattice (owner key per cell,
exact 5^3 sub-cell solid fraction) and runs the fused collide-stream kernel,
which also reduces the hydrodynamic force and torque of every particle
straight into ``demslover.gf.force_fluid / moment_fluid``.

Keyword options beyond the reference signature (defaults reproduce the
reference PSC lattice exactly):
  smagorinsky  "off" (reference PSCLattice3D), "reference" (computeOmega before
               the PSC blend, HybridLattice3D.collide order), or "local"
  body_force   lattice-unit body force added as in ForcedLattice3D (default none)
  storage      "f32" | "f16" | "bf16" population storage (FP32 arithmetic)
  lagged_storage   "f16" with storage="f32": the lagged Smagorinsky state
               (drho, u, omega of the previous collision) in FP16 -- 20 B
               per cell less traffic per step, the lagged values rounded to
               FP16 between steps (the reference keeps them in FP32)
  keep_hydroforce  also store the per-cell hydrodynamic force field
  stress       keep the lagged state that compute_stress() needs (the reference's
               stress diagnostics, lbm_solver3d.py:347-456)
  solid_fraction   "exact" (the reference's 5^3 sub-sample count) or "smooth"
               (a C1 ramp of one lattice spacing across the same effective
               surface, differentiable in the particle positions; used by
               lbdem_taichi_b200.lbdem.adjoint)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _native as N
from ..dem3d.demsolver import DEMSolver
from ..lbm3d.lattice import LatticeEngine, LatticeField, to_ref
from ..lbm3d.lbmutils import CellType  # noqa: F401  (in the module namespace, as the reference module has it)


class PSCLattice3D(LatticeEngine):
    def __init__(self, Nx, Ny, Nz, omega, dx, dt, rho, demslover: DEMSolver, *, smagorinsky="off",
                 body_force=None, storage="f32", keep_hydroforce=False, skip_inlet=False,
                 solid_fraction="exact", stress=False, lagged_storage=None):
        super().__init__(Nx, Ny, Nz, omega, dx, dt, rho, smagorinsky=smagorinsky, body_force=body_force,
                         storage=storage, skip_inlet=skip_inlet, stress=stress, lagged_storage=lagged_storage)
        if solid_fraction not in ("exact", "smooth"):
            raise ValueError('solid_fraction must be "exact" or "smooth"')
        self.dem = demslover
        self.solid_fraction = solid_fraction
        nc = self.ncells
        dev = "cuda"
        n = max(demslover.n, 1)
        self._key = torch.zeros(nc, dtype=torch.int32, device=dev)
        self._table = torch.zeros((n, 16), dtype=torch.float32, device=dev)
        self._prev = torch.zeros((n, 4), dtype=torch.float64, device=dev)
        self._hydro = torch.zeros((3, nc), dtype=torch.float32, device=dev) if keep_hydroforce else None
        self._psc = N.Psc()
        p = self._psc
        p.dx, p.dt, p.rho_unit = float(dx), float(dt), float(rho)
        dom = demslover.config.domain
        p.xmin, p.ymin, p.zmin = float(dom.xmin), float(dom.ymin), float(dom.zmin)
        p.skip_inlet = int(skip_inlet)
        p.key, p.table, p.prev = N.ptr(self._key), N.ptr(self._table), N.ptr(self._prev)
        p.have_prev = 0
        p.hydro_out = N.ptr(self._hydro)
        # map reuse: a bed whose particles did not move keeps its exact owner
        # keys (the check runs on the device; the cell types must not have changed)
        self._map_moved = torch.zeros(2, dtype=torch.int32, device=dev)
        p.map_moved = N.ptr(self._map_moved)
        p.map_reuse, p.map_parity = 0, 0
        self._mapped_epoch = -1
        # periodic axes of the DEM domain (image shift = domain length / dx): used by the
        # pipelined run, and for periodic images in the DEM solver's "wrapped" mode
        self.wrapped = getattr(demslover, "compat", "reference") == "wrapped"
        if self.wrapped and solid_fraction == "smooth":
            raise ValueError('the smooth solid fraction has no periodic images (DEMSolver compat="wrapped")')
        dom = demslover.config.domain
        lens = (dom.xmax - dom.xmin, dom.ymax - dom.ymin, dom.zmax - dom.zmin)
        for a in range(3):
            per = demslover.config.boundaryType[2 * a] == demslover.config.BOUNDARY_TYPE_PERIODIC
            p.periodic[a] = int(per)
            p.period[a] = float(lens[a] / dx) if per else 0.0
            p.wrap[a] = int(per and self.wrapped)
        p.disp_limit = 0.0
        # pipelined run(): near-block mask, side stream for the DEM and the next map
        self.pipeline_margin = 0.25
        self._pipeline_choice = None      # run(pipeline="auto"): measured on the first long run
        self._hcounts = None              # pipelined run: list lengths read back (pinned host memory)
        self._pipeline_probe = None       # (sequential, pipelined) ms per step of that measurement
        self._near = None
        self._side = None
        self._clear_stream = None
        if solid_fraction == "smooth":
            self._eps = torch.zeros(nc, dtype=torch.float32, device=dev)
            self._map_scratch = torch.zeros(nc, dtype=torch.int64, device=dev)
            p.eps = N.ptr(self._eps)
        else:
            self._eps = None
            p.eps = None
        self._grains = N.Grains()
        g, t = self._grains, demslover._t
        g.n = demslover.n
        g.pos, g.radius, g.vel, g.omega = (N.ptr(t["position"]), N.ptr(t["radius"]), N.ptr(t["velocity"]),
                                           N.ptr(t["omega"]))
        g.force_fluid, g.moment_fluid = N.ptr(t["force_fluid"]), N.ptr(t["moment_fluid"])
        shp = (self.Nx, self.Ny, self.Nz)
        self._decoded = None
        self.id = LatticeField(self, "id", shp, np.int32, lambda: self._decode_fields()[0])
        self.volfrac = LatticeField(self, "volfrac", shp, np.float64, lambda: self._decode_fields()[1])
        self.weight = LatticeField(self, "weight", shp, np.float64, lambda: self._decode_fields()[2])
        self.velsolid = LatticeField(self, "velsolid", shp + (3,), np.float64, lambda: self._decode_fields()[3])
        self.hydroforce = LatticeField(self, "hydroforce", shp + (3,), np.float64, self._pull_hydro)

    # ------------------------------------------------------------ fields
    def _decode_fields(self):
        if self._decoded is None:
            nc = self.ncells
            dev = "cuda"
            idt = torch.empty(nc, dtype=torch.int32, device=dev)
            vf = torch.empty(nc, dtype=torch.float32, device=dev)
            w = torch.empty(nc, dtype=torch.float32, device=dev)
            vs = torch.empty((3, nc), dtype=torch.float32, device=dev)
            psc = C.byref(self._psc) if self.dem.n > 0 else None
            N.call("lbdem_psc_decode", C.byref(self._lat), psc, N.ptr(idt), N.ptr(vf), N.ptr(w), N.ptr(vs),
                   N.stream_handle())
            sh = (self.Nz, self.Ny, self.Nx)
            self._decoded = (to_ref(idt.cpu().numpy().reshape(sh)),
                             to_ref(vf.cpu().numpy().reshape(sh).astype(np.float64)),
                             to_ref(w.cpu().numpy().reshape(sh).astype(np.float64)),
                             to_ref(vs.cpu().numpy().reshape((3,) + sh).astype(np.float64)))
        return self._decoded

    def _pull_hydro(self):
        if self._hydro is None:
            raise RuntimeError("construct PSCLattice3D(..., keep_hydroforce=True) to keep the per-cell force")
        return to_ref(self._hydro.cpu().numpy().reshape(3, self.Nz, self.Ny, self.Nx).astype(np.float64))

    def _invalidate_views(self):
        super()._invalidate_views()
        self._decoded = None
        for fld in ("id", "volfrac", "weight", "velsolid", "hydroforce"):
            if hasattr(self, fld):
                getattr(self, fld).invalidate()

    # ------------------------------------------------------------ coupling
    def grains2lattice(self):
        """Map the particles onto the lattice (psclattice3d.py:84-182)."""
        if self.dem.n == 0:
            return
        self._sync_inputs()
        if self.solid_fraction == "smooth":
            N.call("lbdem_psc_map_smooth", C.byref(self._lat), C.byref(self._psc), C.byref(self._grains),
                   N.ptr(self._map_scratch), N.stream_handle())
        else:
            self._psc.map_reuse = int(self._mapped_epoch == self._links_epoch)
            N.call("lbdem_psc_map", C.byref(self._lat), C.byref(self._psc), C.byref(self._grains),
                   N.stream_handle())
            self._mapped_epoch = self._links_epoch
        self._decoded = None

    def initialize(self):
        """f = feq(rho, vel); map the grains (psclattice3d.py:60-78)."""
        super().initialize()
        self.grains2lattice()
        self._invalidate_views()

    def collide(self):
        """Map grains, PSC/BGK collision and force reduction (psclattice3d.py:187-218),
        fused with the pending stream."""
        self.grains2lattice()
        if self._hydro is not None:
            self._hydro.zero_()
        if self.dem.n > 0:
            self._launch_step(C.byref(self._psc), C.byref(self._grains))
        else:
            self._launch_step()

    def step(self, sub_cycles: int = 1):
        """One coupled time step: collide(); stream(); DEM x sub_cycles
        (the driver loop of single_particle_settle.py:230-241)."""
        self.collide()
        self.stream()
        self.dem.run_substeps(sub_cycles)

    def run(self, n_steps: int, sub_cycles: int = 1, pipeline="auto"):
        """n_steps coupled steps (step() n times).  Pipelined, the step's
        x-blocks that no particle can reach -- at most ``pipeline_margin``
        lattice units of motion per step, 0.25 by default -- are streamed and
        collided on the GPU while the DEM sub-steps and the next map still run
        on a second stream; the blocks near particles follow once the map is
        ready.  Every cell is computed once from the same inputs, so the result
        is the sequential loop's (force sums may differ in the last FP64 bits:
        they are added atomically).  A particle that moves farther than the
        margin in one step raises a lattice fault at the next check_status().

        ``pipeline``: True, False, or "auto" (default): the first call of at
        least 32 steps times twelve sequential and twelve pipelined steps and
        keeps the faster form for this lattice (the pipeline pays where the DEM
        and the map are a large part of the step and particles leave much of
        the lattice free).  Lattices without particles, with the smooth solid
        fraction, with periodic images or beyond 8192 x 4096 x 4096 cells always
        run sequentially."""
        n = int(n_steps)
        if n <= 0:
            return
        # block-list entries pack z, y and the x-block into 12 + 12 + 8 bits
        eligible = (self.dem.n > 0 and self.solid_fraction == "exact" and not self.wrapped
                    and self.Nx <= 8192 and self.Ny <= 4096 and self.Nz <= 4096)
        if pipeline == "auto":
            if not eligible:
                pipeline = False
            elif self._pipeline_choice is None and n >= 32:
                def timed(fn):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    fn()
                    e1.record()
                    e1.synchronize()
                    return e0.elapsed_time(e1)
                # untimed first: the first launches of either form's kernels load their code
                self._run_pipelined(2, sub_cycles)
                self._run_sequential(2, sub_cycles)
                t_seq = timed(lambda: self._run_sequential(12, sub_cycles)) / 12
                t_pipe = timed(lambda: self._run_pipelined(12, sub_cycles)) / 12
                self._pipeline_choice = t_pipe < t_seq
                self._pipeline_probe = (t_seq, t_pipe)
                n -= 28
                pipeline = self._pipeline_choice
            else:
                pipeline = bool(self._pipeline_choice)
        if not pipeline or not eligible or n < 2:
            self._run_sequential(n, sub_cycles)
            return
        self._run_pipelined(n, sub_cycles)

    def _run_sequential(self, n: int, sub_cycles: int):
        """step() n times.  Where particles move (so the map cannot be reused),
        the owner keys of each step's map but the last are cleared on a second
        stream beside the DEM sub-steps (lbdem_psc_map_clear) instead of by the
        next map: the step kernel is their last reader, and the next map then
        claims on clear keys."""
        early = (n > 1 and self.dem.n > 0 and self.solid_fraction == "exact"
                 and bool((self.dem._t["freeze"] == 0).any()))
        if not early:
            for _ in range(n):
                self.step(sub_cycles)
            return
        S = torch.cuda.current_stream()
        if self._clear_stream is None:
            self._clear_stream = torch.cuda.Stream()   # default priority: the DEM's blocks are not held back
        D = self._clear_stream
        lat, psc, grains = C.byref(self._lat), C.byref(self._psc), C.byref(self._grains)
        for k in range(n):
            self.collide()
            self.stream()
            stepped = torch.cuda.Event()
            stepped.record(S)
            self.dem.run_substeps(sub_cycles)
            if k < n - 1:
                with torch.cuda.stream(D):
                    D.wait_event(stepped)
                    N.call("lbdem_psc_map_clear", lat, psc, grains, D.cuda_stream)
                    cleared = torch.cuda.Event()
                    cleared.record(D)
                S.wait_event(cleared)

    def _side_stream(self):
        if self._side is None:
            self._side = torch.cuda.Stream(priority=-1)
        return self._side

    def _run_pipelined(self, n: int, sub_cycles: int):
        S = torch.cuda.current_stream()
        if self._near is None:
            self._side_stream()
            nblk = self.Ny * self.Nz * self._nb
            self._near = torch.zeros(nblk, dtype=torch.uint8, device="cuda")
            # two block lists: the side stream builds the next step's while this step's is in use
            self._blocks = [torch.zeros(nblk, dtype=torch.int32, device="cuda") for _ in range(2)]
            self._bcounts = [torch.zeros(2 + 2 * ((nblk + 1023) // 1024), dtype=torch.int32, device="cuda")
                             for _ in range(2)]
        D = self._side
        lat, psc, grains = C.byref(self._lat), C.byref(self._psc), C.byref(self._grains)
        d = self.dem._d
        sync = d.sync
        d.sync = None                      # no grid-wide DEM launch: its blocks share the GPU with the step
        self._psc.disp_limit = float(self.pipeline_margin)

        nblk = self._near.numel()
        if self._hcounts is None:
            # list lengths read back asynchronously: each phase launch is sized from the latest one
            # that has arrived (a launch beside it takes any entries beyond), not from all blocks
            self._hcounts = torch.zeros((4, 2), dtype=torch.int32).pin_memory()
            self._hcount_ev = [None] * 4
        slot = [0]

        def near_blocks(buf, stream):
            # blocks a particle can reach before the DEM moves it (current positions)
            N.call("lbdem_psc_near_blocks", lat, psc, grains, float(self.pipeline_margin), N.ptr(self._near),
                   N.ptr(self._blocks[buf]), N.ptr(self._bcounts[buf]), stream.cuda_stream)
            i = slot[0] % 4
            with torch.cuda.stream(stream):
                self._hcounts[i].copy_(self._bcounts[buf][:2], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
            self._hcount_ev[i] = (slot[0], ev)
            slot[0] += 1

        def estimate():
            # (far, near) list lengths of the newest read-back that has completed, with 3 % + 64 headroom
            best = None
            for rec in self._hcount_ev:
                if rec is not None and (best is None or rec[0] > best[0]) and rec[1].query():
                    best = rec
            if best is None:
                return 0, 0
            far, near = (int(v) for v in self._hcounts[best[0] % 4])
            pad = lambda c: c + c // 32 + 64 if c + c // 32 + 64 < nblk else 0  # noqa: E731
            return pad(far), pad(near)

        try:
            self.collide()                 # step 0: map and full fused step
            self.stream()
            near_blocks(0, S)
            lists = None                   # event: the next step's lists are built (side stream)
            for k in range(n):
                last = k == n - 1
                buf = k & 1
                ev = torch.cuda.Event()
                ev.record(S)
                with torch.cuda.stream(D):
                    D.wait_event(ev)
                    self.dem.run_substeps(sub_cycles)
                    if not last:
                        self.grains2lattice()      # map of step k+1
                    mapped = torch.cuda.Event()
                    mapped.record(D)
                    if k < n - 2:
                        near_blocks(1 - buf, D)    # the next iteration's lists, from the positions of this map
                        nxt = torch.cuda.Event()
                        nxt.record(D)
                if last:
                    S.wait_event(mapped)
                    break
                if lists is not None:
                    S.wait_event(lists)
                lists = nxt if k < n - 2 else None
                src = self._cur
                blk = (N.ptr(self._blocks[buf]), N.ptr(self._bcounts[buf]))
                far_n, near_n = estimate()
                N.call("lbdem_psc_step_phase", lat, psc, grains, src, 1 - src, 1, *blk, far_n, S.cuda_stream)
                S.wait_event(mapped)
                if self._hydro is not None:
                    self._hydro.zero_()
                N.call("lbdem_psc_step_phase", lat, psc, grains, src, 1 - src, 2, *blk, near_n, S.cuda_stream)
                self._cur, self._cur_kind, self._collided = 1 - src, "fpc", None
        finally:
            d.sync = sync
            self._psc.disp_limit = 0.0
        self._invalidate_views()
