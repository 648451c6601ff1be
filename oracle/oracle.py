"""ctypes front end of the FP64 C restatement in ``lbdem_oracle.c``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg as the parity checker / CPU baseline.
The product (``lbdem_taichi_b200``) never imports this module.

Arrays keep the reference's shapes: lattice fields (Nx, Ny, Nz[, k]) with k
fastest (Taichi dense layout), particle fields (n, ...).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lbdem_oracle.c")
LIB = os.path.join(HERE, "_build", "liboracle.so")

CT_FLUID, CT_OBSTACLE, CT_VEL_LADD = 1, 8, 32


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (OpenMP, strict IEEE: no contraction)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
               "-o", LIB, SRC, "-lm"]
        subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        for fn in ("orc_initialize", "orc_collide", "orc_stream"):
            getattr(_lib, fn).argtypes = [C.c_void_p]
        _lib.orc_grains2lattice.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_grains2lattice_all.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_lattice2grains.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_global_sums.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_dem_run_simulation.argtypes = [C.c_void_p]
        _lib.orc_dem_candidates.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        _lib.orc_dem_candidates.restype = C.c_int
        _lib.orc_map_smooth.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_compute_stress.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_adjoint_collide.argtypes = [C.c_void_p] + [C.c_void_p] * 5 + [C.c_int]
        _lib.orc_adjoint_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_pos_adjoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class _Lat(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("omega0", C.c_double), ("dx", C.c_double), ("dt", C.c_double), ("rho_unit", C.c_double),
                ("smag_cs", C.c_double), ("smag", C.c_int), ("psc", C.c_int), ("force_on", C.c_int),
                ("force", C.c_double * 3), ("skip_inlet", C.c_int),
                ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
                ("ct", C.c_void_p), ("f", C.c_void_p), ("fpc", C.c_void_p), ("feq", C.c_void_p),
                ("rho", C.c_void_p), ("vel", C.c_void_p), ("omega", C.c_void_p), ("id", C.c_void_p),
                ("volfrac", C.c_void_p), ("weight", C.c_void_p), ("velsolid", C.c_void_p),
                ("hydroforce", C.c_void_p)]


class _Grains(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", C.c_void_p), ("radius", C.c_void_p), ("vel", C.c_void_p),
                ("omega", C.c_void_p), ("force_fluid", C.c_void_p), ("moment_fluid", C.c_void_p)]


class OracleLattice:
    """FP64 lattice with the reference's fields and step functions.

    ``smag``: apply ``computeOmega`` (lbm_solver3d.py:500-513) before
    ``compute_feq`` -- BasicLattice3D.collide / HybridLattice3D.collide order.
    ``psc``: PSC weighted collision (psclattice3d.py:240-261).
    ``force``: ForcedLattice3D source term (lbm_foecelover.py:52-68).
    """

    def __init__(self, nx, ny, nz, omega0, dx=1.0, dt=1.0, rho_unit=1.0, smag_cs=0.1, smag=False,
                 psc=False, force=None, skip_inlet=False, dom_min=(0.0, 0.0, 0.0)):
        self.shape = (nx, ny, nz)
        s = self.shape
        self.ct = np.full(s, CT_FLUID, np.int32)
        self.f = np.zeros(s + (19,))
        self.fpc = np.zeros(s + (19,))
        self.feq = np.zeros(s + (19,))
        self.rho = np.ones(s)
        self.vel = np.zeros(s + (3,))
        self.omega = np.full(s, float(omega0))
        self.id = np.full(s, -1, np.int32)
        self.volfrac = np.zeros(s)
        self.weight = np.zeros(s)
        self.velsolid = np.zeros(s + (3,))
        self.hydroforce = np.zeros(s + (3,))
        self.p = _Lat()
        p = self.p
        p.nx, p.ny, p.nz = nx, ny, nz
        p.omega0, p.dx, p.dt, p.rho_unit = omega0, dx, dt, rho_unit
        p.smag_cs, p.smag, p.psc = smag_cs, int(bool(smag)), int(bool(psc))
        p.force_on = int(force is not None)
        if force is not None:
            p.force[:] = [float(v) for v in force]
        p.skip_inlet = int(bool(skip_inlet))
        p.xmin, p.ymin, p.zmin = [float(v) for v in dom_min]

    def _bind(self):
        p = self.p
        for name in ("ct", "f", "fpc", "feq", "rho", "vel", "omega", "id", "volfrac", "weight",
                     "velsolid", "hydroforce"):
            a = getattr(self, name)
            assert a.flags.c_contiguous
            setattr(p, name, a.ctypes.data)
        return C.byref(p)

    def initialize(self):
        lib().orc_initialize(self._bind())

    def collide(self):
        lib().orc_collide(self._bind())

    def stream(self):
        lib().orc_stream(self._bind())

    def grains2lattice(self, g: "OracleGrains"):
        """psclattice3d.py:84-182, each cell visiting only the grains listed
        for its bin (identical to ``grains2lattice_all``)."""
        lib().orc_grains2lattice(self._bind(), g._bind())

    def grains2lattice_all(self, g: "OracleGrains"):
        """psclattice3d.py:84-182 as written: every cell visits every grain."""
        lib().orc_grains2lattice_all(self._bind(), g._bind())

    def lattice2grains(self, g: "OracleGrains"):
        lib().orc_lattice2grains(self._bind(), g._bind())

    def global_sums(self):
        out = np.zeros(4)
        lib().orc_global_sums(self._bind(), _p(out))
        return out

    def compute_stress(self):
        """(Nx, Ny, Nz, 7): xx, yy, zz, xy, xz, yz, shear magnitude (lbm_solver3d.py:347-404);
        zero on skipped cells as the reference's fields."""
        out = np.zeros(self.shape + (7,))
        lib().orc_compute_stress(self._bind(), _p(out))
        self.stress = out
        return out

    def plane_average_stress(self, axis, position):
        """lbm_solver3d.py:406-456: mean (xy, xz, yz) stress over the FLUID cells of a plane."""
        sl = [slice(None)] * 3
        sl[axis] = position
        fl = (self.ct[tuple(sl)] & CT_FLUID) != 0
        st = self.stress[tuple(sl)]
        n = int(fl.sum())
        if n == 0:
            return np.zeros(3)
        return np.array([st[..., 3][fl].sum() / n, st[..., 4][fl].sum() / n, st[..., 5][fl].sum() / n])

    # reverse mode on a frozen bed (smooth solid fraction)
    def map_smooth(self, g: "OracleGrains"):
        lib().orc_map_smooth(self._bind(), g._bind())

    def adjoint_collide(self, lam, sbar, bbar, gbar, loss_dir, seed):
        d = np.ascontiguousarray(loss_dir, np.float64)
        lib().orc_adjoint_collide(self._bind(), _p(lam), _p(sbar), _p(bbar), _p(gbar), _p(d), int(seed))

    def adjoint_stream(self, sbar, lam_prev):
        lib().orc_adjoint_stream(self._bind(), _p(sbar), _p(lam_prev))

    def pos_adjoint(self, g: "OracleGrains", bbar, pos_bar):
        lib().orc_pos_adjoint(self._bind(), g._bind(), _p(bbar), _p(pos_bar))


class OracleGrains:
    def __init__(self, pos, radius, vel, omega):
        self.pos = np.ascontiguousarray(pos, np.float64)
        self.radius = np.ascontiguousarray(radius, np.float64)
        self.vel = np.ascontiguousarray(vel, np.float64)
        self.omega = np.ascontiguousarray(omega, np.float64)
        n = len(self.radius)
        self.force_fluid = np.zeros((n, 3))
        self.moment_fluid = np.zeros((n, 3))
        self.g = _Grains()

    def _bind(self):
        g = self.g
        g.n = len(self.radius)
        for name in ("pos", "radius", "vel", "omega", "force_fluid", "moment_fluid"):
            setattr(g, name, getattr(self, name).ctypes.data)
        return C.byref(g)


class _Dem(C.Structure):
    _fields_ = [("n", C.c_int), ("maxc", C.c_int), ("model", C.c_int), ("dt", C.c_double),
                ("g", C.c_double * 3), ("dom_min", C.c_double * 3), ("dom_max", C.c_double * 3),
                ("periodic", C.c_int * 3), ("bp_min", C.c_double * 3), ("cell_size", C.c_double),
                ("table_size", C.c_int),
                ("E", C.c_double * 2), ("nu", C.c_double * 2), ("mu", C.c_double * 2),
                ("e", C.c_double * 2), ("kn", C.c_double * 2), ("ks", C.c_double * 2),
                ("dpn", C.c_double * 2), ("dps", C.c_double * 2)] + \
               [(n, C.c_void_p) for n in ("pos", "vel", "acc", "force", "quat", "omega", "omega_dot",
                                          "moment", "inertia", "mass", "radius", "force_fluid",
                                          "moment_fluid", "freeze", "fixvel", "cf_i", "cf_j",
                                          "cf_active", "cfn", "cf_shear", "cf_pos", "cf_force",
                                          "wcf_active", "wcf_shear", "wcf_pos", "wcf_force")] + \
               [("wall_n", C.c_double * 18), ("wall_d", C.c_double * 6), ("wall_periodic", C.c_int32 * 6)] + \
               [(n, C.c_void_p) for n in ("ht_offset", "ht_count", "ht_current", "pid", "bits")] + \
               [("status", C.c_int32)]


def next_pow2(x: int) -> int:
    """bpcd/utils.py:12-19"""
    x -= 1
    for s in (1, 2, 4, 8, 16):
        x |= x >> s
    return x + 1


def bpcd_table_size(n_unused, max_radius, dmin, dmax):
    """bpcd.py:48-65"""
    v = (np.asarray(dmax, float) - np.asarray(dmin, float)) / (4.0 * max_radius)
    size = int(v[0] * v[1] * v[2])
    size = next_pow2(next_pow2(size))
    return min(max(size, 1 << 20), 1 << 22)


class OracleDEM:
    """FP64 DEM with the reference's state layout (DEMSolver fields)."""

    def __init__(self, pos, vel, radius, mass, *, dt, gravity, domain, periodic=(False, False, False),
                 model="hertz", E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3, pp_mu=0.3, pw_mu=0.3,
                 pp_e=0.9, pw_e=0.9, kn=0.0, ks=0.0, dpn=0.0, max_coord=16, omega=None,
                 bp_min=None, bp_max=None, freeze=None):
        n = len(radius)
        self.n = n
        self.pos = np.ascontiguousarray(pos, np.float64).copy()
        self.vel = np.ascontiguousarray(vel, np.float64).copy()
        self.radius = np.ascontiguousarray(radius, np.float64).copy()
        self.mass = np.ascontiguousarray(mass, np.float64).copy()
        self.acc = np.zeros((n, 3))
        self.force = np.zeros((n, 3))
        self.quat = np.zeros((n, 4))
        self.quat[:, 0] = 1.0
        self.omega = np.zeros((n, 3)) if omega is None else np.ascontiguousarray(omega, np.float64).copy()
        self.omega_dot = np.zeros((n, 3))
        self.moment = np.zeros((n, 3))
        self.inertia = np.zeros((n, 3, 3))
        for i in range(n):
            self.inertia[i] = 2.0 / 5.0 * self.mass[i] * self.radius[i] * self.radius[i] * np.eye(3)
        self.force_fluid = np.zeros((n, 3))
        self.moment_fluid = np.zeros((n, 3))
        self.freeze = np.zeros(n, np.int32) if freeze is None else np.asarray(freeze, np.int32).copy()
        self.fixvel = np.zeros(n, np.int32)
        self.maxc = int(max_coord)
        nm = max(n * self.maxc, 1)
        self.cf_i = np.zeros(nm, np.int32)
        self.cf_j = np.zeros(nm, np.int32)
        self.cf_active = np.zeros(nm, np.int32)
        self.cfn = np.zeros(n, np.int32)
        self.cf_shear = np.zeros((nm, 3))
        self.cf_pos = np.zeros((nm, 3))
        self.cf_force = np.zeros((nm, 3))
        self.wcf_active = np.zeros((n, 6), np.int32)
        self.wcf_shear = np.zeros((n, 6, 3))
        self.wcf_pos = np.zeros((n, 6, 3))
        self.wcf_force = np.zeros((n, 6, 3))
        xmin, xmax, ymin, ymax, zmin, zmax = [float(v) for v in domain]
        bp_min = (xmin, ymin, zmin) if bp_min is None else bp_min
        bp_max = (xmax, ymax, zmax) if bp_max is None else bp_max
        rmax = float(self.radius.max())
        T = bpcd_table_size(n, rmax, bp_min, bp_max)
        self.ht_offset = np.zeros(T, np.int32)
        self.ht_count = np.zeros(T, np.int32)
        self.ht_current = np.zeros(T, np.int32)
        self.pid = np.zeros(max(n, 1), np.int32)
        self.bits = np.zeros(max(n * n, 1), np.uint8)
        d = _Dem()
        self.d = d
        d.n, d.maxc = n, self.maxc
        d.model = 0 if model == "hertz" else 1
        d.dt = dt
        d.g[:] = list(map(float, gravity))
        d.dom_min[:] = [xmin, ymin, zmin]
        d.dom_max[:] = [xmax, ymax, zmax]
        d.periodic[:] = [int(bool(v)) for v in periodic]
        d.bp_min[:] = list(map(float, bp_min))
        d.cell_size = rmax * 4.0
        d.table_size = T
        d.E[:] = [E, wall_E]
        d.nu[:] = [nu, wall_nu]
        d.mu[:] = [pp_mu, pw_mu]
        d.e[:] = [pp_e, pw_e]
        d.kn[:] = [kn, 0.0]
        d.ks[:] = [ks, 0.0]
        d.dpn[:] = [dpn, 0.0]
        d.dps[:] = [0.0, 0.0]   # demsolver.py:250 writes dp_tratio, a member Material lacks
        d.wall_n[:] = [1.0, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, -1.0]
        d.wall_d[:] = [xmax, -xmin, ymax, -ymin, zmax, -zmin]
        d.wall_periodic[:] = [int(bool(periodic[w // 2])) for w in range(6)]

    def _bind(self):
        d = self.d
        names = ("pos", "vel", "acc", "force", "quat", "omega", "omega_dot", "moment", "inertia", "mass",
                 "radius", "force_fluid", "moment_fluid", "freeze", "fixvel", "cf_i", "cf_j", "cf_active",
                 "cfn", "cf_shear", "cf_pos", "cf_force", "wcf_active", "wcf_shear", "wcf_pos", "wcf_force",
                 "ht_offset", "ht_count", "ht_current", "pid", "bits")
        for nm in names:
            a = getattr(self, nm)
            assert a.flags.c_contiguous, nm
            setattr(d, nm, a.ctypes.data)
        return C.byref(d)

    @property
    def status(self):
        return int(self.d.status)

    def run_simulation(self):
        lib().orc_dem_run_simulation(self._bind())

    def candidates(self):
        cap = max(64, self.n * 64)
        out = np.zeros((cap, 2), np.int32)
        m = lib().orc_dem_candidates(self._bind(), _p(out), cap)
        assert m <= cap
        return out[:m].copy()

    def active_pairs(self):
        """{(i, j): shear} for every active particle-particle contact."""
        res = {}
        for i in range(self.n):
            for o in range(min(int(self.cfn[i]), self.maxc)):
                s = i * self.maxc + o
                if self.cf_active[s]:
                    res[(int(self.cf_i[s]), int(self.cf_j[s]))] = self.cf_shear[s].copy()
        return res


def frozen_bed_drag(shape, omega0, ct, radius, pos, force, n_steps, loss_dir=(1.0, 0.0, 0.0), grad=False,
                    dx=1.0, dt=1.0, rho_unit=1.0, dom_min=(0.0, 0.0, 0.0)):
    """FP64 drag on a frozen bed after ``n_steps`` PSC steps with the smooth
    solid fraction: L = e . sum_particles force_fluid after the last collide
    (the forward of lbdem_taichi_b200.lbdem.adjoint, restated with the
    reference's own collide / stream / lattice2grains in this file).

    Returns L, or (L, dL/dF (3,), dL/dpos (n, 3)) with ``grad`` (FP64 adjoint;
    every streamed state is kept, so use small lattices)."""
    nx, ny, nz = shape
    lat = OracleLattice(nx, ny, nz, omega0, dx=dx, dt=dt, rho_unit=rho_unit, psc=True, force=force,
                        dom_min=dom_min)
    lat.ct[...] = ct
    n = len(radius)
    g = OracleGrains(pos, radius, np.zeros((n, 3)), np.zeros((n, 3)))
    lat.map_smooth(g)
    lat.initialize()
    e = np.asarray(loss_dir, np.float64)
    states = []
    for step in range(1, n_steps + 1):
        if grad:
            states.append(lat.f.copy())
        lat.collide()
        lat.lattice2grains(g)
        if step < n_steps:
            lat.stream()
    L = float((g.force_fluid.sum(axis=0) * e).sum())
    if not grad:
        return L
    lam = np.zeros_like(lat.f)
    sbar = np.zeros_like(lat.f)
    bbar = np.zeros(shape)
    gbar = np.zeros(3)
    for step in range(n_steps, 0, -1):
        lat.f[...] = states[step - 1]
        lat.adjoint_collide(None if step == n_steps else lam, sbar, bbar, gbar, e, step == n_steps)
        if step > 1:
            lat.adjoint_stream(sbar, lam)
    pos_bar = np.zeros((n, 3))
    lat.pos_adjoint(g, bbar, pos_bar)
    return L, gbar, pos_bar
