"""ctypes bindings of liblbdem.so (declarations in include/lbdem.h).

The library is the only compute path: if it is missing, or no CUDA device is
present, every solver call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblbdem.so")

LBDEM_OK = 0
LBDEM_ERR_ARG, LBDEM_ERR_LAUNCH, LBDEM_ERR_UNSUPPORTED = 1, 2, 3
ST_NAN, ST_RHO, ST_VELMAX = 1, 2, 4
ST_CONTACT_OVERFLOW, ST_GRID_OVERFLOW, ST_GID_OVERFLOW, ST_CELL_OVERFLOW = 8, 16, 32, 64
ST_WAIT_TIMEOUT = 128
ST_PIPELINE_MARGIN = 256
ABI_VERSION = 4        # LBDEM_ABI_VERSION of include/lbdem.h
F32, F16, BF16 = 0, 1, 2
LINK_FLUID = 1 << 20   # LBDEM_LINK_FLUID: the link mask of every cell of an all-FLUID lattice
SMAG_OFF, SMAG_REFERENCE, SMAG_LOCAL = 0, 1, 2
SUM_BLOCKS = 1184
SUM_PARTIALS = 4 * SUM_BLOCKS

STATUS_TEXT = {
    ST_NAN: "non-finite population or moment",
    ST_RHO: "fluid density <= 0",
    ST_VELMAX: "fluid speed reached sqrt(2/3) (lattice Mach limit)",
    ST_CONTACT_OVERFLOW: "contact count exceeds max_coordinate_number",
    ST_GRID_OVERFLOW: "particle left the broad-phase grid",
    ST_GID_OVERFLOW: "too many particles for the PSC owner key",
    ST_CELL_OVERFLOW: "a broad-phase cell holds more particles than its list capacity",
    ST_WAIT_TIMEOUT: "a bounded wait for an asynchronous copy gave up",
    ST_PIPELINE_MARGIN: "a particle moved farther in one step than the pipelined run's margin",
}

vp = C.c_void_p


class Lattice(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("storage", C.c_int32),
                ("omega0", C.c_float), ("smag_cs", C.c_float), ("smag_mode", C.c_int32),
                ("force_on", C.c_int32), ("force", C.c_float * 3), ("scale16", C.c_float),
                ("f", vp * 2), ("rho", vp), ("vel", vp), ("aux", vp), ("links", vp),
                ("status", vp), ("moving", vp), ("ct", vp), ("bnd_cells", vp), ("bnd_na", C.c_uint32),
                ("bnd_nb", C.c_uint32), ("bnd_f0", vp), ("bnd_slip", C.c_int32), ("stress", vp), ("links_all", C.c_uint32),
                ("aux_half", C.c_int32)]


class Grains(C.Structure):
    _fields_ = [("n", C.c_int32), ("pos", vp), ("radius", vp), ("vel", vp), ("omega", vp),
                ("force_fluid", vp), ("moment_fluid", vp)]


class Psc(C.Structure):
    _fields_ = [("dx", C.c_double), ("dt", C.c_double), ("rho_unit", C.c_double),
                ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
                ("skip_inlet", C.c_int32), ("key", vp), ("table", vp), ("prev", vp),
                ("have_prev", C.c_int32), ("hydro_out", vp), ("eps", vp), ("map_moved", vp),
                ("map_reuse", C.c_int32), ("map_parity", C.c_int32), ("wrap", C.c_int32 * 3),
                ("period", C.c_double * 3), ("periodic", C.c_int32 * 3), ("disp_limit", C.c_double)]


_DEM_PTRS = ("pos", "vel", "acc", "force", "quat", "omega", "omega_dot", "moment", "inertia", "mass", "radius",
             "force_fluid", "moment_fluid", "freeze", "fixvel", "cf_j", "cf_active", "cfn", "cf_add", "cf_shear", "cf_pos",
             "cf_force", "wcf_active", "wcf_shear", "wcf_pos", "wcf_force")


class Dem(C.Structure):
    _fields_ = [("n", C.c_int32), ("maxc", C.c_int32), ("model", C.c_int32),
                ("dt", C.c_double), ("g", C.c_double * 3), ("dom_min", C.c_double * 3),
                ("dom_max", C.c_double * 3), ("periodic", C.c_int32 * 3), ("bp_min", C.c_double * 3),
                ("cell_size", C.c_double), ("gdim", C.c_int32 * 3),
                ("E", C.c_double * 2), ("nu", C.c_double * 2), ("mu", C.c_double * 2), ("e", C.c_double * 2),
                ("kn", C.c_double * 2), ("ks", C.c_double * 2), ("dpn", C.c_double * 2), ("dps", C.c_double * 2),
                ("wall_n", C.c_double * 18), ("wall_d", C.c_double * 6), ("wall_periodic", C.c_int32 * 6)] + \
               [(n, vp) for n in _DEM_PTRS] + \
               [("cell_cap", C.c_int32), ("cell_count", vp), ("cell_list", vp), ("acc_force", vp),
                ("acc_moment", vp), ("parity", C.c_int32), ("status", vp), ("sync", vp),
                ("wrap_pairs", C.c_int32)]


EXPORTS = {
    "lbdem_abi_version": ([], C.c_int),
    "lbdem_last_error": ([], C.c_char_p),
    "lbdem_build_links": ([vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp], C.c_int),
    "lbdem_lattice_init": ([vp, C.c_int32, vp], C.c_int),
    "lbdem_psc_map": ([vp, vp, vp, vp], C.c_int),
    "lbdem_psc_step_f32": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp], C.c_int),
    "lbdem_psc_step_f16": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp], C.c_int),
    "lbdem_psc_step_bf16": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp], C.c_int),
    "lbdem_stream_moments": ([vp, C.c_int32, C.c_int32, vp], C.c_int),
    "lbdem_psc_decode": ([vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "lbdem_dem_bin": ([vp, vp], C.c_int),
    "lbdem_dem_substeps": ([vp, C.c_int32, vp], C.c_int),
    "lbdem_global_sums_f64": ([vp, C.c_int32, vp, vp, vp], C.c_int),
    "lbdem_global_sums_f64_noalloc": ([vp, C.c_int32, vp, vp], C.c_int),
    "lbdem_psc_map_smooth": ([vp, vp, vp, vp, vp], C.c_int),
    "lbdem_dem_launches_last": ([], C.c_int),
    "lbdem_stress": ([vp, C.c_int32, vp, vp], C.c_int),
    "lbdem_psc_step_adjoint_f32": ([vp, vp, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, vp], C.c_int),
    "lbdem_psc_force_adjoint": ([vp, vp, vp, vp, vp, vp], C.c_int),
    "lbdem_boundary_cells": ([vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_uint32, vp, vp, vp], C.c_int),
    "lbdem_psc_near_blocks": ([vp, vp, vp, C.c_double, vp, vp, vp, vp], C.c_int),
    "lbdem_psc_step_phase": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_uint32, vp], C.c_int),
    "lbdem_psc_map_clear": ([vp, vp, vp, vp], C.c_int),
}

_lib = None

# kernels launched per call (for the launch count reported by bench.py)
KERNELS_PER_CALL = {"lbdem_build_links": 1, "lbdem_lattice_init": 1, "lbdem_psc_map": 2,
                    "lbdem_psc_step_f32": 1, "lbdem_psc_step_f16": 1, "lbdem_psc_step_bf16": 1,
                    "lbdem_stream_moments": 1, "lbdem_psc_decode": 1, "lbdem_dem_bin": 1,
                    "lbdem_global_sums_f64": 2, "lbdem_global_sums_f64_noalloc": 2,
                    "lbdem_psc_map_smooth": 3, "lbdem_stress": 1, "lbdem_psc_step_adjoint_f32": 1, "lbdem_psc_force_adjoint": 1,
                    "lbdem_boundary_cells": 3, "lbdem_psc_near_blocks": 4, "lbdem_psc_step_phase": 1,
                    "lbdem_psc_map_clear": 1}
# calls followed by the boundary pass: one more kernel per non-empty phase
_BOUNDARY_CALLS = ("lbdem_psc_step_f32", "lbdem_psc_step_f16", "lbdem_psc_step_bf16", "lbdem_stream_moments")
_launches = [0]


def reset_launch_count():
    _launches[0] = 0


def launch_count():
    return _launches[0]


class LbdemError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Load liblbdem.so and declare its C ABI.  Raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LbdemError(f"{path} is missing: build it with `python -m lbdem_taichi_b200.build`")
    lib = C.CDLL(path)
    for name, (args, res) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.lbdem_abi_version() != ABI_VERSION:
        raise LbdemError("liblbdem.so ABI version mismatch")
    _lib = lib
    return lib


def _boundary_phases(arg):
    L = getattr(arg, "_obj", None)
    return int(L.bnd_na > 0) + int(L.bnd_nb > 0) if isinstance(L, Lattice) else 0


def _map_launches(arg):
    # lbdem_psc_map skips its clearing pass when there is nothing to clear or check
    P = getattr(arg, "_obj", None)
    if P is None or P.have_prev or P.disp_limit > 0.0:
        return 2
    return 1


def call(name: str, *args):
    pre = _map_launches(args[1]) if name == "lbdem_psc_map" else None
    rc = getattr(load(), name)(*args)
    if pre is not None:
        _launches[0] += pre
    else:
        _launches[0] += (load().lbdem_dem_launches_last() if name == "lbdem_dem_substeps"
                         else KERNELS_PER_CALL.get(name, 0))
    if name == "lbdem_psc_step_phase" and args[8]:
        _launches[0] += 1     # a launch sized from an estimate is followed by the one that takes the rest
    if name in _BOUNDARY_CALLS or (name == "lbdem_psc_step_phase" and args[5] == 2):
        _launches[0] += _boundary_phases(args[0])
    if rc != LBDEM_OK:
        msg = load().lbdem_last_error().decode(errors="replace")
        raise LbdemError(f"{name} failed (code {rc}): {msg}")
    return rc


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else t.data_ptr()


def stream_handle():
    import torch
    return torch.cuda.current_stream().cuda_stream


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise LbdemError("lbdem_taichi_b200 needs a CUDA device (sm_100a); none is available")
    load()
