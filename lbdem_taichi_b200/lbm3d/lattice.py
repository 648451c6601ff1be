"""D3Q19 lattice on the GPU (API of src/lbm3d/lbm_solver3d.py:17-513 and
src/lbm3d/lbm_foecelover.py:15-68).

Device layout: populations f[buf][q][z][y][x] (x fastest) in two buffers of
the storage type, stored as deviations from the lattice weights; macroscopic
rho/u in FP32; per-cell link masks built once from CellType.  Python-scope
field access uses the reference's index order [i, j, k] = [x, y, z] and
shapes (Nx, Ny, Nz[, k]).

Collide/stream: ``collide()`` launches ONE fused kernel that streams the
pending post-collision populations (pull), takes moments, applies the
collision and writes new post-collision populations; ``stream()`` only marks
them as pending.  Reading populations or moments materialises the stream
(one extra pass) so reads always see the reference's post-stream state.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _native as N
from .lbmutils import CellType, UnitConverter

_STORAGE = {"f32": (N.F32, torch.float32, 1.0), "f16": (N.F16, torch.float16, 4096.0),
            "bf16": (N.BF16, torch.bfloat16, 1.0)}
_SMAG = {"off": N.SMAG_OFF, "reference": N.SMAG_REFERENCE, "local": N.SMAG_LOCAL}
# free-surface cell types (the reference's PSC path never sets them)
_UNSUPPORTED = CellType.INTERFACE | CellType.GAS
# cell types handled by the boundary pass: wet-node rules of the stream's second
# pass (lbm_solver3d.py:242-250) and free-slip walls (whose neighbours it streams)
_OPEN = CellType.VEL_ZOUHE | CellType.VEL_EXIT | CellType.Pre_ZOUHE | CellType.VEL_INLET_LADD | CellType.FREE_SLIP
_FACES = CellType.LEFT | CellType.RIGHT | CellType.BOTTOM | CellType.TOP | CellType.BACK | CellType.FRONT

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
_STRESS_FIELDS = ("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz", "shear_stress_mag")
C_Q = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1],
                [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]], dtype=np.float64)
QINV = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])


def _mirror_table(axis):
    """Index of the direction with c's `axis` component negated (the
    free-slip reflection tables qsyx / qsyy / qsyz, lbm_solver3d.py:50-57)."""
    flip = C_Q.copy()
    flip[:, axis] *= -1
    return np.array([int(np.flatnonzero((C_Q == v).all(axis=1))[0]) for v in flip], dtype=np.int32)


def to_ref(a):
    """device order (..., z, y, x) -> reference order (x, y, z, ...)."""
    a = np.asarray(a)
    if a.ndim == 3:
        return np.ascontiguousarray(a.transpose(2, 1, 0))
    return np.ascontiguousarray(a.transpose(3, 2, 1, 0))


def from_ref(a, comps=None):
    a = np.asarray(a)
    if comps is None:
        return np.ascontiguousarray(a.transpose(2, 1, 0))
    return np.ascontiguousarray(a.transpose(3, 2, 1, 0))


class _CellVector(np.ndarray):
    """One cell's vector of a writable field: component writes
    (``lattice.vel[i, j, k][0] = u``, as Taichi allows) go back to the field."""

    def __setitem__(self, k, v):
        super().__setitem__(k, v)
        self._field[self._idx] = np.asarray(self)


class LatticeField:
    """Reference-shaped view of one lattice field.

    Element writes (``lattice.CT[i, j, k] = ...``) go to a host mirror and are
    uploaded before the next kernel launch; reads download once and are served
    from the mirror until the device changes the field.
    """

    def __init__(self, owner, name, shape, dtype, pull, push=None):
        self._owner, self._name = owner, name
        self._shape, self._dtype = shape, dtype
        self._pull, self._push = pull, push
        self._host = None
        self._dirty = False

    @property
    def shape(self):
        return self._shape

    def _get_host(self):
        if self._host is None:
            self._host = np.asarray(self._pull(), dtype=self._dtype).reshape(self._shape)
        return self._host

    def invalidate(self):
        if not self._dirty:
            self._host = None

    def to_numpy(self):
        return self._get_host().copy()

    def __getitem__(self, idx):
        v = self._get_host()[idx]
        if not isinstance(v, np.ndarray):
            return v
        v = v.copy()
        if self._push is not None and v.ndim == 1 and len(self._shape) == 4 and isinstance(idx, tuple) \
                and len(idx) == 3 and all(isinstance(i, (int, np.integer)) for i in idx):
            v = v.view(_CellVector)
            v._field, v._idx = self, idx
        return v

    def _writable(self):
        if self._push is None:
            raise AttributeError(f"field '{self._name}' is read-only")
        h = self._get_host()
        self._dirty = True
        self._owner._host_dirty(self._name)
        return h

    def __setitem__(self, idx, v):
        self._writable()[idx] = v

    def fill(self, v):
        self._writable()[...] = v

    def from_numpy(self, a):
        self._writable()[...] = np.asarray(a).reshape(self._shape)

    def flush(self):
        if self._dirty:
            self._push(self._host)
            self._dirty = False


class LatticeEngine:
    """Device state + kernels shared by BasicLattice3D / ForcedLattice3D / PSCLattice3D."""
    D = 3
    Q = 19
    c = C_Q
    w = W
    qinv = QINV
    qsyx, qsyy, qsyz = _mirror_table(0), _mirror_table(1), _mirror_table(2)
    cssq = 1.0 / 3.0
    velmax = (2.0 / 3.0) ** 0.5
    SmagorinskyConstant = 0.1

    def __init__(self, Nx, Ny, Nz, omega, dx, dt, rho, *, smagorinsky="off", body_force=None,
                 storage="f32", skip_inlet=True, stress=False, lagged_storage=None):
        N.require_cuda()
        if storage not in _STORAGE:
            raise ValueError(f"storage must be one of {sorted(_STORAGE)}")
        if lagged_storage not in (None, storage) and (storage, lagged_storage) != ("f32", "f16"):
            raise ValueError('lagged_storage: "f16" under storage="f32" (or the storage form itself)')
        if smagorinsky not in _SMAG:
            raise ValueError(f"smagorinsky must be one of {sorted(_SMAG)}")
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.omega0 = float(omega)
        self.unit = UnitConverter(dx, dt, rho)
        self.storage = storage
        self.smagorinsky = smagorinsky
        self.skip_inlet = skip_inlet
        kind, tdtype, scale = _STORAGE[storage]
        self._kind, self._tdtype, self._scale = kind, tdtype, scale
        self.body_force = None if body_force is None else np.asarray(body_force, np.float64)
        nc = self.Nx * self.Ny * self.Nz
        self.ncells = nc
        dev = "cuda"
        # populations and lagged Smagorinsky state are blocked by 32 cells
        # along x: [z][y][x // 32][q][x % 32] (x padded to a multiple of 32)
        self._nb = (self.Nx + 31) // 32
        nblk = self.Nz * self.Ny * self._nb
        self._f = [torch.zeros((nblk, 19, 32), dtype=tdtype, device=dev) for _ in range(2)]
        self._rho = torch.ones(nc, dtype=torch.float32, device=dev)
        self._vel = torch.zeros((3, nc), dtype=torch.float32, device=dev)
        # lagged state (drho, u, omega) of the last collision: needed by the
        # reference Smagorinsky form and by the stress diagnostics
        self.stress_enabled = bool(stress) or smagorinsky == "reference"
        # (FP32 storage may keep it in FP16: lagged_storage="f16", 20 B per cell less step traffic)
        self._aux_half = lagged_storage == "f16" and storage == "f32"
        self.lagged_storage = "f16" if self._aux_half else storage
        self._aux = (torch.zeros((nblk, 5, 32), dtype=torch.float16 if self._aux_half else tdtype, device=dev)
                     if self.stress_enabled else None)
        self._stress = None
        self._stress_pending = False   # compute_stress() not evaluated yet (fused into the next collide)
        self._links_all = N.LINK_FLUID   # cell types start as FLUID everywhere: one link mask
        self._links = torch.zeros(nc, dtype=torch.int32, device=dev)
        self._moving = None
        self.has_moving_walls = False
        # open boundaries: cells of the boundary pass (lbdem_boundary_cells)
        self.has_open_boundaries = False
        self._bnd = None
        self._bnd_counts = torch.zeros(2, dtype=torch.int32, device=dev)
        self._bnd_scratch = None
        self._bnd_f0 = None
        self._has_slip = False
        # device cell types start as FLUID, as the reference fills CT (lbm_solver3d.py:136-137)
        self._ct_dev = torch.full((nc,), int(CellType.FLUID), dtype=torch.int32, device=dev)
        self._status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._sum_out = torch.zeros(4, dtype=torch.float64, device=dev)
        self._sum_part = torch.zeros(N.SUM_PARTIALS, dtype=torch.float64, device=dev)
        self._links_dirty = True
        self._links_epoch = 0          # counts link-mask rebuilds (cell-type changes)
        self._initialized = False
        self._cur = 0
        self._cur_kind = "f"
        self._collided = None
        self._macro_valid = True
        self._host_ct = np.full((self.Nx, self.Ny, self.Nz), CellType.FLUID, np.int32)

        shp = (self.Nx, self.Ny, self.Nz)
        self.CT = LatticeField(self, "CT", shp, np.int32, lambda: self._host_ct, self._push_ct)
        self.CT._host = self._host_ct
        self.rho = LatticeField(self, "rho", shp, np.float64, self._pull_rho, self._push_rho)
        self.vel = LatticeField(self, "vel", shp + (3,), np.float64, self._pull_vel, self._push_vel)
        self.f = LatticeField(self, "f", shp + (19,), np.float64, self._pull_f)
        self.omega = LatticeField(self, "omega", shp, np.float64, self._pull_omega)
        for m, name in enumerate(_STRESS_FIELDS):
            setattr(self, name, LatticeField(self, name, shp, np.float64, lambda m=m: self._pull_stress(m)))
        self._lat = N.Lattice()
        self._fill_desc()

    # ------------------------------------------------------------ descriptor
    def _fill_desc(self):
        L = self._lat
        L.nx, L.ny, L.nz = self.Nx, self.Ny, self.Nz
        L.storage = self._kind
        L.omega0 = self.omega0
        L.smag_cs = float(self.SmagorinskyConstant)
        L.smag_mode = _SMAG[self.smagorinsky]
        if self.body_force is not None:
            L.force_on = 1
            L.force[:] = [float(v) for v in self.body_force]
        else:
            L.force_on = 0
        L.scale16 = self._scale
        L.f[0], L.f[1] = N.ptr(self._f[0]), N.ptr(self._f[1])
        L.rho, L.vel = N.ptr(self._rho), N.ptr(self._vel)
        L.aux = N.ptr(self._aux)
        L.aux_half = int(self._aux_half)
        L.links = N.ptr(self._links)
        L.links_all = self._links_all    # one mask for every cell (all FLUID), else 0
        L.status = N.ptr(self._status)
        L.ct = N.ptr(self._ct_dev)

    # ------------------------------------------------------------ host mirrors
    def _host_dirty(self, name):
        if name == "CT":
            self._links_dirty = True

    def _push_ct(self, host):
        bad = np.bitwise_and(host, _UNSUPPORTED)
        if bad.any():
            raise NotImplementedError("free-surface cell types (INTERFACE, GAS) are not supported")
        slip = np.bitwise_and(host, CellType.FREE_SLIP) != 0
        if (slip & (np.bitwise_and(host, _FACES) == 0)).any():
            raise ValueError("FREE_SLIP cells need a face bit (LEFT/RIGHT/BOTTOM/TOP/BACK/FRONT) for the mirror "
                             "direction (lbm_solver3d.py:230-236)")
        self._ct_dev.copy_(torch.from_numpy(from_ref(host.astype(np.int32)).reshape(-1)))
        # an all-FLUID lattice has one link mask everywhere: the step reads none
        self._links_all = N.LINK_FLUID if bool((host == CellType.FLUID).all()) else 0
        self._lat.links_all = self._links_all
        self.has_open_boundaries = bool(np.bitwise_and(host, _OPEN).any())
        self._has_slip = bool(slip.any())
        # moving walls and Ladd inlets: per-cell velocity-link bits, allocated on first use
        if np.bitwise_and(host, CellType.VEL_LADD | CellType.VEL_INLET_LADD).any():
            if self._moving is None:
                self._moving = torch.zeros(self.ncells, dtype=torch.int32, device="cuda")
            self._lat.moving = N.ptr(self._moving)
        else:
            self._lat.moving = None
        self.has_moving_walls = self._lat.moving is not None

    def _build_boundary_list(self):
        """Cells of the boundary pass, in lattice order (one host read of the counts)."""
        L = self._lat
        L.bnd_slip = int(self._has_slip)
        if not self.has_open_boundaries:
            L.bnd_cells, L.bnd_na, L.bnd_nb, L.bnd_f0 = None, 0, 0, None
            return
        if self._bnd_scratch is None:
            self._bnd_scratch = torch.zeros(2 * self.Ny * self.Nz, dtype=torch.int32, device="cuda")
        if self._bnd is None:
            # six faces' worth; grown below when the lattice holds more boundary cells
            n0 = 2 * (self.Ny * self.Nz + self.Nx * self.Nz + self.Nx * self.Ny) + 64
            self._bnd = torch.zeros(n0, dtype=torch.int32, device="cuda")
        for _ in range(2):
            cap = self._bnd.numel()
            N.call("lbdem_boundary_cells", N.ptr(self._links), self.Nx, self.Ny, self.Nz, N.ptr(self._bnd), cap,
                   N.ptr(self._bnd_counts), N.ptr(self._bnd_scratch), N.stream_handle())
            na, nb = (int(v) for v in self._bnd_counts.cpu())
            if na + nb <= cap:
                break
            self._bnd = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
        L.bnd_cells, L.bnd_na, L.bnd_nb = N.ptr(self._bnd), na, nb
        if self._bnd_f0 is None or self._bnd_f0.shape[1] < max(nb, 1):
            self._bnd_f0 = torch.zeros((19, max(nb, 1)), dtype=self._tdtype, device="cuda")
        L.bnd_f0 = N.ptr(self._bnd_f0)

    def _push_rho(self, host):
        self._rho.copy_(torch.from_numpy(from_ref(host).reshape(-1).astype(np.float32)))

    def _push_vel(self, host):
        self._vel.copy_(torch.from_numpy(from_ref(host, 3).reshape(3, -1).astype(np.float32)))

    def _sync_inputs(self):
        if self._stress_pending and (self.CT._dirty or self.rho._dirty or self.vel._dirty):
            # a pending compute_stress() belongs to the state before these writes
            self._flush_stress()
        # the Smagorinsky constant is a class attribute in the reference
        # (lbm_solver3d.py:97, read at :508); drivers may change it on the class or the instance
        self._lat.smag_cs = float(self.SmagorinskyConstant)
        if self.CT._dirty and self._cur_kind == "fpc" and self._collided is None:
            # the reference streams eagerly: a pending stream uses the old cell types
            self._materialize()
        self.CT.flush()
        if self._links_dirty:
            N.call("lbdem_build_links", N.ptr(self._ct_dev), self.Nx, self.Ny, self.Nz, int(self.skip_inlet),
                   N.ptr(self._links), N.ptr(self._moving) if self._lat.moving else None,
                   N.stream_handle())
            self._build_boundary_list()
            self._links_dirty = False
            self._links_epoch += 1
        self.rho.flush()
        self.vel.flush()

    # ------------------------------------------------------------ populations
    def _decode(self, buf):
        # every storage form holds h = (f - w) S / w
        h = self._unblock(self._f[buf], 19)
        return h * (W[:, None] / self._scale) + W[:, None]

    def _unblock(self, t, k):
        """(k, Ncells) FP64 host copy of a blocked [z][y][x//32][k][x%32] buffer."""
        a = t.float().cpu().numpy().astype(np.float64).reshape(self.Nz, self.Ny, self._nb, k, 32)
        a = a.transpose(3, 0, 1, 2, 4).reshape(k, self.Nz, self.Ny, self._nb * 32)[..., :self.Nx]
        return a.reshape(k, -1)

    def _materialize(self):
        """Bring the lattice to the reference's post-stream state on the device."""
        if self._collided is not None:
            src, dst, gather = self._collided
            if gather:
                raise RuntimeError("populations between collide() and stream() are not resident; "
                                   "read them after stream()")
            return src
        if self._cur_kind == "fpc":
            src = self._cur
            N.call("lbdem_stream_moments", C.byref(self._lat), src, 1 - src, N.stream_handle())
            self._cur = 1 - src
            self._cur_kind = "f"
            self._macro_valid = True
        return self._cur

    def _pull_f(self):
        buf = self._materialize()
        d = self._decode(buf).reshape(19, self.Nz, self.Ny, self.Nx)
        return to_ref(d)

    def _pull_rho(self):
        self._materialize()
        return to_ref(self._rho.cpu().numpy().reshape(self.Nz, self.Ny, self.Nx).astype(np.float64))

    def _pull_vel(self):
        self._materialize()
        return to_ref(self._vel.cpu().numpy().reshape(3, self.Nz, self.Ny, self.Nx).astype(np.float64))

    def _pull_omega(self):
        if self._aux is None:
            return np.full((self.Nx, self.Ny, self.Nz), self.omega0)
        om = self._unblock(self._aux, 5)[4].reshape(self.Nz, self.Ny, self.Nx)
        ct = self._host_ct
        out = to_ref(om)
        skip = (ct & (CellType.OBSTACLE | CellType.VEL_LADD | CellType.FREE_SLIP | CellType.VEL_INLET_LADD)) != 0
        out[skip] = self.omega0
        return out

    def _invalidate_views(self):
        for fld in (self.rho, self.vel, self.f, self.omega):
            fld.invalidate()

    # ------------------------------------------------------------ diagnostics
    def compute_stress(self):
        """Stress tensor and shear magnitude of the current (post-stream) state
        (lbm_solver3d.py:347-404): sigma = -(1 - omega/2) sum c c (f - feq),
        feq and omega of the last collision.  Needs the lagged state: construct
        the lattice with stress=True (implied by smagorinsky="reference").

        The result is that of the state at this call.  It is evaluated lazily:
        the next collide() gathers exactly this state, so it writes the stress
        as an optional output of the fused step (no extra pass over the
        populations -- the reference's drivers call compute_stress() after
        every stream); reading a stress field, a plane average, changing a
        field or restoring a state first evaluates it in a pass of its own.
        Lattices with open boundaries (boundary-pass cells) evaluate it at once."""
        if not self.stress_enabled:
            raise RuntimeError("construct the lattice with stress=True to keep the state compute_stress needs")
        self._sync_inputs()
        if self._stress is None:
            self._stress = torch.zeros((7, self.ncells), dtype=torch.float32, device="cuda")
        self._stress_pending = True
        if self.has_open_boundaries or self._collided is not None:
            self._flush_stress()
        for name in _STRESS_FIELDS:
            getattr(self, name).invalidate()

    def _flush_stress(self):
        """Evaluate a pending compute_stress() now, in a pass of its own."""
        if not self._stress_pending:
            return
        self._stress_pending = False
        buf = self._materialize()
        N.call("lbdem_stress", C.byref(self._lat), buf, N.ptr(self._stress), N.stream_handle())
        for name in _STRESS_FIELDS:
            getattr(self, name).invalidate()

    def _pull_stress(self, m):
        self._flush_stress()
        if self._stress is None:
            return np.zeros((self.Nx, self.Ny, self.Nz))
        return to_ref(self._stress[m].cpu().numpy().reshape(self.Nz, self.Ny, self.Nx).astype(np.float64))

    def compute_plane_average_stress(self, axis: int, position: int):
        """Mean (xy, xz, yz) stress over the FLUID cells of the plane normal to
        `axis` at index `position` (lbm_solver3d.py:406-456); zeros for an
        empty plane.  Uses the stress of the last compute_stress()."""
        self._flush_stress()
        if self._stress is None:
            return np.zeros(3)
        st = self._stress.view(7, self.Nz, self.Ny, self.Nx)
        ct = self._ct_dev.view(self.Nz, self.Ny, self.Nx)
        # reference axis 0/1/2 = x/y/z; device arrays are [z][y][x]
        dim = 2 - int(axis)
        sel = [slice(None)] * 3
        sel[dim] = int(position)
        fl = (ct[tuple(sel)] & CellType.FLUID) != 0
        n = int(fl.sum().item())
        if n == 0:
            return np.zeros(3)
        out = torch.stack([st[k][tuple(sel)][fl].double().sum() for k in (3, 4, 5)]) / n
        return out.cpu().numpy()

    # ------------------------------------------------------------ restart
    def state_dict(self):
        """Post-stream populations (storage form, blocked layout), density,
        velocity and the lagged Smagorinsky state, as host copies, for a
        restart (the reference saves no populations).  Taken between steps;
        a pending stream is applied first."""
        if not self._initialized:
            raise RuntimeError("initialize() the lattice before taking its state")
        self._sync_inputs()
        buf = self._materialize()
        d = {"shape": (self.Nx, self.Ny, self.Nz), "storage": self.storage, "smagorinsky": self.smagorinsky,
             "lagged_storage": self.lagged_storage,
             "omega0": self.omega0, "f": self._f[buf].detach().cpu().clone(),
             "rho": self._rho.detach().cpu().clone(), "vel": self._vel.detach().cpu().clone()}
        if self._aux is not None:
            d["aux"] = self._aux.detach().cpu().clone()
        return d

    def load_state_dict(self, d):
        if tuple(d["shape"]) != (self.Nx, self.Ny, self.Nz) or d["storage"] != self.storage:
            raise ValueError("restart state is for another lattice size or storage form")
        if d["smagorinsky"] != self.smagorinsky:
            raise ValueError("restart state was taken with another Smagorinsky mode")
        self._flush_stress()
        self._sync_inputs()
        # both buffers: cells no collision writes (walls, skipped inlets) and a
        # Ladd inlet's populations must read the same from either
        self._f[0].copy_(d["f"])
        self._f[1].copy_(d["f"])
        self._rho.copy_(d["rho"])
        self._vel.copy_(d["vel"])
        if self._aux is not None:
            self._aux.copy_(d["aux"])
        self.rho.invalidate()
        self.vel.invalidate()
        self._cur, self._cur_kind, self._collided = 0, "f", None
        self._initialized = True
        self._invalidate_views()

    def save_state(self, path):
        torch.save(self.state_dict(), path)

    def load_state(self, path):
        self.load_state_dict(torch.load(path, weights_only=True))

    # ------------------------------------------------------------ kernels
    def initialize(self):
        """f = feq(rho, vel) on updated cells (lbm_solver3d.py:157-171)."""
        self._flush_stress()
        self._sync_inputs()
        N.call("lbdem_lattice_init", C.byref(self._lat), 0, N.stream_handle())
        self._cur, self._cur_kind, self._collided = 0, "f", None
        self._initialized = True
        self._invalidate_views()

    def _step_fn(self):
        return {N.F32: "lbdem_psc_step_f32", N.F16: "lbdem_psc_step_f16", N.BF16: "lbdem_psc_step_bf16"}[self._kind]

    def _launch_step(self, psc=None, grains=None):
        if not self._initialized:
            raise RuntimeError("call initialize() before collide()")
        self._sync_inputs()
        if self._collided is not None:
            src, dst, gather = self._collided
        else:
            src, dst, gather = self._cur, 1 - self._cur, int(self._cur_kind == "fpc")
        ev = getattr(self, "_kernel_events", None)
        fused_stress = self._stress_pending
        if fused_stress:
            # the step gathers the state of the pending compute_stress(): it writes the stress too
            self._lat.stress = N.ptr(self._stress)
        if ev:
            ev[0].record()
        try:
            N.call(self._step_fn(), C.byref(self._lat), psc, grains, src, dst, gather, N.stream_handle())
        finally:
            if fused_stress:
                self._lat.stress = None
                self._stress_pending = False
        if ev:
            ev[1].record()
        self._collided = (src, dst, gather)
        self._invalidate_views()

    def collide(self):
        self._launch_step()

    def stream(self):
        """Streaming (lbm_solver3d.py:197-250); the fused kernel performs it at
        the next collide() or when populations/moments are read."""
        if self._collided is None:
            raise RuntimeError("stream() must follow collide()")
        _, dst, _ = self._collided
        self._cur, self._cur_kind, self._collided = dst, "fpc", None
        self._invalidate_views()

    def global_sums(self):
        """FP64 [mass, momentum_x, momentum_y, momentum_z] of the updated cells."""
        self._sync_inputs()
        buf = self._collided[0] if self._collided is not None else self._cur
        N.call("lbdem_global_sums_f64", C.byref(self._lat), buf, N.ptr(self._sum_out), N.ptr(self._sum_part),
               N.stream_handle())
        return self._sum_out.cpu().numpy().copy()

    def check_status(self):
        s = int(self._status.item())
        if s:
            bits = [txt for b, txt in N.STATUS_TEXT.items() if s & b]
            raise N.LbdemError("lattice fault: " + "; ".join(bits))

    def clear_status(self):
        self._status.zero_()


class BasicLattice3D(LatticeEngine):
    """BGK + Smagorinsky lattice (BasicLattice3D.collide, lbm_solver3d.py:176-192:
    computeOmega with the previous step's feq and omega, then BGK)."""

    def __init__(self, Nx, Ny, Nz, omega, dx, dt, rho, *, storage="f32", smagorinsky="reference", stress=False,
                 lagged_storage=None):
        super().__init__(Nx, Ny, Nz, omega, dx, dt, rho, smagorinsky=smagorinsky, storage=storage,
                         skip_inlet=True, stress=stress, lagged_storage=lagged_storage)


class ForcedLattice3D(LatticeEngine):
    """BGK with the simple body-force term w_q rho (c_q . F)/cs^2
    (lbm_foecelover.py:15-68).  F is a physical acceleration."""

    def __init__(self, Nx, Ny, Nz, omega, dx, dt, rho, F, *, storage="f32"):
        unit = UnitConverter(dx, dt, rho)
        super().__init__(Nx, Ny, Nz, omega, dx, dt, rho, smagorinsky="off",
                         body_force=unit.getLbAccel(np.asarray(F, np.float64)), storage=storage, skip_inlet=False)
        self.F = self.body_force
