"""DEMSolver with device-resident FP64 state (API of
src/dem3d/demsolver/demsolver.py:24-862).

Particle state lives in torch CUDA tensors laid out like the reference's Grain
fields ((n, 3) rows); ``run_simulation`` launches the sm_100a sub-step kernels
(broad phase, contacts, walls, integration) through liblbdem.so.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
import warnings

import numpy as np
import torch

from .. import _native as N
from .demconfig import DEMSolverConfig, HertzContactConfig, LinearContactConfig
from .p4io import read_p4p, write_p4c, write_p4p

DEV = "cuda"


def next_pow2(x: int) -> int:
    """bpcd/utils.py:12-19"""
    x -= 1
    for s in (1, 2, 4, 8, 16):
        x |= x >> s
    return x + 1


def reference_table_size(max_radius, dmin, dmax) -> int:
    """Hash-table size the reference broad phase would use (bpcd.py:48-65)."""
    v = (np.asarray(dmax, float) - np.asarray(dmin, float)) / (4.0 * max_radius)
    size = next_pow2(next_pow2(int(v[0] * v[1] * v[2])))
    return min(max(size, 1 << 20), 1 << 22)


class _Member:
    """One member of the grain field (``gf.position`` etc.)."""

    def __init__(self, owner, name, tensor, np_dtype=None):
        self._owner, self._name, self._t = owner, name, tensor
        self._np_dtype = np_dtype

    @property
    def shape(self):
        return tuple(self._t.shape)

    def to_numpy(self):
        a = self._t.detach().cpu().numpy()
        return a.astype(self._np_dtype) if self._np_dtype is not None else a

    def from_numpy(self, a):
        self._t.copy_(torch.as_tensor(np.asarray(a).reshape(self._t.shape), dtype=self._t.dtype))
        self._owner._touched(self._name)

    def fill(self, v):
        self._t[...] = torch.as_tensor(np.asarray(v), dtype=self._t.dtype)
        self._owner._touched(self._name)

    def __getitem__(self, i):
        return self._t[i].detach().cpu().numpy()

    def __setitem__(self, i, v):
        self._t[i] = torch.as_tensor(np.asarray(v), dtype=self._t.dtype)
        self._owner._touched(self._name)


class _Elem:
    """``gf[i]``: attribute access to particle i."""

    def __init__(self, gf, i):
        object.__setattr__(self, "_gf", gf)
        object.__setattr__(self, "_i", int(i))

    def __getattr__(self, name):
        m = self._gf._members.get(name)
        if m is None:
            raise AttributeError(name)
        v = m._t[self._i].detach().cpu().numpy()
        return v.item() if v.ndim == 0 else v

    def __setattr__(self, name, v):
        m = self._gf._members.get(name)
        if m is None:
            raise AttributeError(f"Grain has no member {name}")
        m[self._i] = v


class GrainField:
    """Struct-of-arrays view matching the reference's ``gf`` (grain.py:23-52)."""

    def __init__(self, solver, members):
        self._solver = solver
        self._members = members

    @property
    def shape(self):
        return (self._solver.n,)

    def __getattr__(self, name):
        m = self.__dict__.get("_members", {}).get(name)
        if m is None:
            raise AttributeError(name)
        return m

    def __getitem__(self, i):
        return _Elem(self, i)


class DEMSolver:
    """``compat="reference"`` (default) reproduces the reference: the broad
    phase never proposes a pair across a periodic face and PSC lattices built
    on this solver map a sphere without its periodic images (bpcd.py:154-194,
    psclattice3d.py:102-108).  ``compat="wrapped"`` adds the periodic images in
    both (contacts across periodic faces; spheres that cross them are mapped on
    both sides, with minimum-image lever arms); every periodic length must span
    at least four broad-phase cells (4 x 4 r_max)."""

    def __init__(self, config: DEMSolverConfig, *, compat: str = "reference"):
        if compat not in ("reference", "wrapped"):
            raise ValueError('compat must be "reference" or "wrapped"')
        self.compat = compat
        self.config = config
        self.contact_model = None
        self.n = 0
        self.gf = None

    # ------------------------------------------------------------------ setup
    def init_particle_fields(self, file_name: str, domain_min, domain_max):
        """Read a p4p file (demsolver.py:130-309: single-space separated,
        1-based IDs) and allocate the device state."""
        N.require_cuda()
        p = read_p4p(file_name)
        self._allocate(p["ID"], p["group"], p["radius"], p["mass"], p["pos"], p["vel"], p["density"], domain_min,
                       domain_max)

    def init_particle_arrays(self, radius, mass, pos, vel, domain_min, domain_max, ID=None, group=None):
        """Same as init_particle_fields, from arrays instead of a p4p file."""
        N.require_cuda()
        radius = np.asarray(radius, np.float64)
        n = len(radius)
        ID = np.arange(1, n + 1) if ID is None else np.asarray(ID)
        group = np.zeros(n, np.int64) if group is None else np.asarray(group)
        mass = np.asarray(mass, np.float64)
        density = 3 * mass[-1] / (4 * math.pi * radius[-1] ** 3) if n else 0.0
        self._allocate(ID, group, radius, mass, np.asarray(pos, np.float64), np.asarray(vel, np.float64), density,
                       domain_min, domain_max)

    def _allocate(self, ID, group, radius, mass, pos, vel, density, domain_min, domain_max):
        cfg = self.config
        n = len(radius)
        self.n = n
        f64 = dict(dtype=torch.float64, device=DEV)
        i32 = dict(dtype=torch.int32, device=DEV)
        t = {}
        t["ID"] = torch.as_tensor(ID, dtype=torch.int64, device=DEV)
        t["groupID"] = torch.as_tensor(group, dtype=torch.int64, device=DEV)
        t["materialType"] = torch.zeros(n, **i32)
        t["radius"] = torch.as_tensor(radius, **f64)
        t["mass"] = torch.as_tensor(mass, **f64)
        t["position"] = torch.as_tensor(pos.reshape(n, 3), **f64).contiguous()
        t["velocity"] = torch.as_tensor(vel.reshape(n, 3), **f64).contiguous()
        for k in ("acceleration", "force", "omega", "omega_dot", "moment", "force_fluid", "moment_fluid"):
            t[k] = torch.zeros((n, 3), **f64)
        t["quaternion"] = torch.zeros((n, 4), **f64)
        t["quaternion"][:, 0] = 1.0
        inertia = np.zeros((n, 3, 3))
        for i in range(n):
            inertia[i] = 2.0 / 5.0 * mass[i] * radius[i] * radius[i] * np.eye(3)
        t["inertia"] = torch.as_tensor(inertia, **f64)
        t["freeze"] = torch.zeros(n, **i32)
        t["fixvel"] = torch.zeros(n, **i32)
        self._t = t
        members = {k: _Member(self, k, v) for k, v in t.items()}
        members["freeze"]._np_dtype = bool
        members["fixvel"]._np_dtype = bool
        self.gf = GrainField(self, members)

        maxc = int(cfg.particle_props.max_coordinate_number)
        self.maxc = maxc
        ns = max(n * maxc, 1)
        self.cf_j = torch.zeros(ns, **i32)
        self.cf_active = torch.zeros(ns, **i32)
        self.cfn = torch.zeros(max(n, 1), **i32)
        self.cf_add = torch.zeros(max(n, 1), **i32)
        self.cf_shear = torch.zeros((ns, 3), **f64)
        self.cf_pos = torch.zeros((ns, 3), **f64)
        self.cf_force = torch.zeros((ns, 3), **f64)
        self.wcf_active = torch.zeros((max(n, 1), 6), **i32)
        self.wcf_shear = torch.zeros((max(n, 1), 6, 3), **f64)
        self.wcf_pos = torch.zeros((max(n, 1), 6, 3), **f64)
        self.wcf_force = torch.zeros((max(n, 1), 6, 3), **f64)
        self.status = torch.zeros(1, **i32)

        # broad phase: the reference's cell size and origin, dense grid
        dmin = np.asarray(domain_min, np.float64)
        dmax = np.asarray(domain_max, np.float64)
        rmax = float(radius.max()) if n else 1.0
        self.max_radius = rmax
        self.cell_size = rmax * 4.0
        ext = np.floor((dmax - dmin) / self.cell_size).astype(int)
        gdim = ext + 4          # reference cells -1 .. ext+2
        self.gdim = gdim
        ncell = int(np.prod(gdim))
        # list capacity of a broad-phase cell: the most spheres of the smallest
        # diameter a cube of edge cell_size can hold at random close packing
        # (0.64), doubled, at least 16
        rmin = float(radius.min()) if n else rmax
        cap = int(np.ceil(2.0 * 0.64 * self.cell_size ** 3 / (4.0 / 3.0 * np.pi * rmin ** 3)))
        self.cell_cap = int(min(max(16, cap), 1024))
        self.cell_count = torch.zeros(2 * ncell, **i32)
        self.cell_list = torch.zeros(ncell * self.cell_cap, **i32)
        self.acc_force = torch.zeros((max(n, 1), 3), **f64)
        self.acc_moment = torch.zeros((max(n, 1), 3), **f64)
        self.sync = torch.zeros(2, **i32)
        # the reference hashes cells into a 2^k table: distinct cells alias when
        # their coordinates agree in the low bits kept by Morton-code mod 2^k
        T = reference_table_size(rmax, dmin, dmax) if n else 1 << 20
        self.reference_table_size = T
        k = T.bit_length() - 1
        nbits = [len([p for p in range(k) if p % 3 == a]) for a in range(3)]
        self.hash_alias_possible = any(int(gdim[a]) > (1 << min(nbits[a], 10)) for a in range(3))
        if self.hash_alias_possible:
            warnings.warn("broad-phase grid spans more cells than the reference's hash keeps apart; "
                          "the reference may propose extra candidate pairs here")

        d = N.Dem()
        self._d = d
        d.n, d.maxc = n, maxc
        d.dt = cfg.dt
        d.g[:] = [float(v) for v in cfg.gravity]
        dom = cfg.domain
        d.dom_min[:] = [dom.xmin, dom.ymin, dom.zmin]
        d.dom_max[:] = [dom.xmax, dom.ymax, dom.zmax]
        d.periodic[:] = [int(cfg.boundaryType[2 * a] == cfg.BOUNDARY_TYPE_PERIODIC) for a in range(3)]
        d.bp_min[:] = [float(v) for v in dmin]
        d.cell_size = self.cell_size
        d.gdim[:] = [int(v) for v in gdim]
        d.wall_n[:] = [float(v) for nrm in cfg.wall_normals for v in nrm]
        d.wall_d[:] = [float(v) for v in cfg.wall_distances]
        d.wall_periodic[:] = [int(b == cfg.BOUNDARY_TYPE_PERIODIC) for b in cfg.boundaryType]
        d.wrap_pairs = int(self.compat == "wrapped")
        self._set_materials(density)
        for name, ten in (("pos", t["position"]), ("vel", t["velocity"]), ("acc", t["acceleration"]),
                          ("force", t["force"]), ("quat", t["quaternion"]), ("omega", t["omega"]),
                          ("omega_dot", t["omega_dot"]), ("moment", t["moment"]), ("inertia", t["inertia"]),
                          ("mass", t["mass"]), ("radius", t["radius"]), ("force_fluid", t["force_fluid"]),
                          ("moment_fluid", t["moment_fluid"]), ("freeze", t["freeze"]), ("fixvel", t["fixvel"]),
                          ("cf_j", self.cf_j), ("cf_active", self.cf_active), ("cfn", self.cfn), ("cf_add", self.cf_add),
                          ("cf_shear", self.cf_shear), ("cf_pos", self.cf_pos), ("cf_force", self.cf_force),
                          ("wcf_active", self.wcf_active), ("wcf_shear", self.wcf_shear),
                          ("wcf_pos", self.wcf_pos), ("wcf_force", self.wcf_force),
                          ("cell_count", self.cell_count), ("cell_list", self.cell_list),
                          ("acc_force", self.acc_force), ("acc_moment", self.acc_moment)):
            setattr(d, name, N.ptr(ten))
        d.cell_cap = self.cell_cap
        d.parity = 0
        d.status = N.ptr(self.status)
        d.sync = N.ptr(self.sync)
        self._binned = False

    # ---------------------------------------------------------------- restart
    _STATE_EXTRA = ("cf_j", "cf_active", "cfn", "cf_add", "cf_shear", "cf_pos", "cf_force", "wcf_active", "wcf_shear",
                    "wcf_pos", "wcf_force", "acc_force", "acc_moment")

    def state_dict(self):
        """Complete particle and contact state (host copies) for a restart; the
        reference keeps no restart state, only its p4p/p4c frames."""
        d = {"grain." + k: v.detach().cpu().clone() for k, v in self._t.items()}
        for k in self._STATE_EXTRA:
            d["contact." + k] = getattr(self, k).detach().cpu().clone()
        d["n"] = self.n
        d["maxc"] = self.maxc
        return d

    def load_state_dict(self, d):
        if int(d["n"]) != self.n or int(d["maxc"]) != self.maxc:
            raise ValueError("restart state is for a different particle count or contact capacity")
        for k, v in self._t.items():
            v.copy_(d["grain." + k])
        for k in self._STATE_EXTRA:
            getattr(self, k).copy_(d["contact." + k])
        self.status.zero_()
        self._binned = False   # the broad-phase lists are rebuilt from the restored positions

    def save_state(self, path):
        torch.save(self.state_dict(), path)

    def load_state(self, path):
        self.load_state_dict(torch.load(path, weights_only=True))

    def _set_materials(self, density):
        """Material table (demsolver.py:222-290): [0] particles, [1] walls."""
        cfg, d = self.config, self._d
        m = cfg.contact_model
        pp, wp = cfg.particle_props, cfg.wall_props
        d.E[:] = [pp.elastic_modulus, wp.elastic_modulus]
        d.nu[:] = [pp.poisson_ratio, wp.poisson_ratio]
        self.material_density = density
        if isinstance(m, LinearContactConfig):
            d.kn[:] = [m.stiffness_normal, 0.0]
            d.ks[:] = [m.stiffness_tangential, 0.0]
            d.dpn[:] = [m.damping_normal, 0.0]
            # demsolver.py:250 assigns the tangential damping to `dp_tratio`, a
            # member the Material struct does not have, so the shear damping
            # ratio the linear law reads (dp_sratio) stays 0.
            d.dps[:] = [0.0, 0.0]
            d.mu[:] = [m.pp_friction, m.pw_friction]
            d.e[:] = [getattr(m, "pp_restitution", 0.0), getattr(m, "pw_restitution", 0.0)]
        elif isinstance(m, HertzContactConfig):
            d.e[:] = [m.pp_restitution, m.pw_restitution]
            d.mu[:] = [m.pp_friction, m.pw_friction]
            d.kn[:] = [0.0, 0.0]
            d.ks[:] = [0.0, 0.0]
            d.dpn[:] = [0.0, 0.0]
            d.dps[:] = [0.0, 0.0]
        else:
            raise ValueError(f"Unknown contact model type: {type(m).__name__}. "
                             f"Expected LinearContactConfig or HertzContactConfig.")

    def set_contact_model(self, model_type: str = "hertz"):
        """Select the contact law; must match the configured model (demsolver.py:311-347)."""
        mt = model_type.lower()
        if mt == "hertz":
            if not isinstance(self.config.contact_model, HertzContactConfig):
                raise ValueError(f"Requested 'hertz' model but config uses "
                                 f"{type(self.config.contact_model).__name__}.")
            self._d.model = 0
        elif mt == "linear":
            if not isinstance(self.config.contact_model, LinearContactConfig):
                raise ValueError(f"Requested 'linear' model but config uses "
                                 f"{type(self.config.contact_model).__name__}.")
            self._d.model = 1
        else:
            raise ValueError(f"Unknown contact model type: '{model_type}'. Valid options are 'hertz' or 'linear'.")
        self.contact_model = mt

    def _touched(self, name):
        if name in ("position", "radius"):
            self._binned = False

    # ---------------------------------------------------------------- stepping
    def _ensure_binned(self):
        if not self._binned:
            N.call("lbdem_dem_bin", C.byref(self._d), N.stream_handle())
            self._binned = True

    def run_substeps(self, nsub: int):
        """``nsub`` consecutive calls of run_simulation, launched back to back."""
        if self.contact_model is None:
            raise RuntimeError("call set_contact_model() before run_simulation()")
        if self.n == 0 or nsub <= 0:
            return
        self._ensure_binned()
        N.call("lbdem_dem_substeps", C.byref(self._d), int(nsub), N.stream_handle())

    def run_simulation(self):
        """One DEM time step (demsolver.py:848-862)."""
        self.run_substeps(1)

    def check_status(self):
        """Raise if the device flagged a fault (reads one int32; synchronises)."""
        s = int(self.status.item())
        if s:
            bits = [txt for b, txt in N.STATUS_TEXT.items() if s & b]
            raise N.LbdemError("DEM fault: " + "; ".join(bits))

    # ------------------------------------------------------------------ output
    def active_contacts(self):
        """{(i, j): (position, force_a, shear)} of active particle-particle contacts."""
        act = self.cf_active.cpu().numpy().astype(bool)
        idx = np.nonzero(act)[0]
        j = self.cf_j.cpu().numpy()
        pos, fa, sh = self.cf_pos.cpu().numpy(), self.cf_force.cpu().numpy(), self.cf_shear.cpu().numpy()
        return {(int(s // self.maxc), int(j[s])): (pos[s], fa[s], sh[s]) for s in idx}

    def save(self, time_: float):
        out_dir = "output"
        os.makedirs(out_dir, exist_ok=True)
        idx = int(round(time_ / self.config.dt))
        name = os.path.join(out_dir, f"output_T{idx:06d}")
        with open(name + ".p4p", "w", encoding="UTF-8") as p4p, open(name + ".p4c", "w", encoding="UTF-8") as p4c:
            self.save_single(p4p, p4c, time_)

    def save_single(self, p4pfile, p4cfile, t: float):
        """Append one p4p/p4c frame (demsolver.py:59-128 format)."""
        tk1 = time.time()
        g = self.gf
        ID = g.ID.to_numpy()
        write_p4p(p4pfile, t, ID, g.groupID.to_numpy(), g.radius.to_numpy(), g.mass.to_numpy(),
                  g.position.to_numpy(), g.velocity.to_numpy())
        # contact rows by (P1, P2): the reference's slot order follows the
        # order of atomic appends, which no run fixes
        con = self.active_contacts()
        write_p4c(p4cfile, t, [[ID[i], ID[j], *p, *f] for (i, j), (p, f, _) in sorted(con.items())])
        print(f"save time cost = {time.time() - tk1:.3f}s")
