"""The C ABI without a GPU: the library loads, exports every function that
include/lbdem.h declares, rejects bad arguments on the host, and the ctypes
descriptors used by the Python classes have the C structs' layout (sizes and
member offsets compiled from the header with gcc)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbdem.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(lbdem_\w+)\s*\(", src, flags=re.M)))


def test_every_declared_function_is_exported():
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    names = _declared()
    assert len(names) >= 15, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the bindings, and vice versa
    assert set(names) == set(N.EXPORTS), set(names) ^ set(N.EXPORTS)
    assert lib.lbdem_abi_version() == N.ABI_VERSION == 4


def test_host_side_argument_checks():
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    assert lib.lbdem_psc_step_f32(None, None, None, 0, 1, 1, None) == N.LBDEM_ERR_ARG
    assert lib.lbdem_last_error()
    L = N.Lattice()
    L.nx, L.ny, L.nz = 8, 8, 8
    L.storage, L.omega0, L.scale16 = N.F32, 1.6, 1.0
    L.links, L.status = 8, 8                             # never dereferenced: checks come first
    assert lib.lbdem_psc_step_f32(C.byref(L), None, None, 0, 0, 1, None) == N.LBDEM_ERR_ARG   # src == dst
    L.smag_mode = N.SMAG_REFERENCE                       # needs the aux buffer
    assert lib.lbdem_psc_step_f32(C.byref(L), None, None, 0, 1, 1, None) == N.LBDEM_ERR_ARG
    L.smag_mode = N.SMAG_OFF
    L.storage = N.F16
    L.scale16 = 0.0                                      # 16-bit forms need a positive scale
    assert lib.lbdem_psc_step_f16(C.byref(L), None, None, 0, 1, 1, None) == N.LBDEM_ERR_ARG
    L.nx, L.ny, L.nz = 2048, 2048, 64                    # 19 * padded cells >= 2^32
    L.scale16 = 4096.0
    assert lib.lbdem_psc_step_f16(C.byref(L), None, None, 0, 1, 1, None) == N.LBDEM_ERR_ARG
    assert b"32-bit" in lib.lbdem_last_error()
    # the adjoint covers FP32 storage with Smagorinsky off only
    P = N.Psc()
    L.nx, L.ny, L.nz, L.storage = 8, 8, 8, N.F16
    d3 = (C.c_double * 3)(1, 0, 0)
    rc = lib.lbdem_psc_step_adjoint_f32(C.byref(L), C.byref(P), 8, None, 8, 8, 8, d3, 1, 1, None)
    assert rc == N.LBDEM_ERR_UNSUPPORTED
    # ... and fixed walls only: open boundaries are refused
    L.storage = N.F32
    L.bnd_na, L.bnd_nb = 4, 0
    rc = lib.lbdem_psc_step_adjoint_f32(C.byref(L), C.byref(P), 8, None, 8, 8, 8, d3, 1, 1, None)
    assert rc == N.LBDEM_ERR_UNSUPPORTED
    # a boundary pass needs the cell types, the list and the macroscopic fields
    assert lib.lbdem_psc_step_f32(C.byref(L), None, None, 0, 1, 1, None) == N.LBDEM_ERR_ARG
    assert b"open boundaries" in lib.lbdem_last_error()
    # the list builder validates its arguments before any launch
    assert lib.lbdem_boundary_cells(None, 8, 8, 8, None, 0, 8, 8, None) == N.LBDEM_ERR_ARG
    assert lib.lbdem_boundary_cells(8, 8, 8, 8, None, 16, 8, 8, None) == N.LBDEM_ERR_ARG   # capacity, no array
    # block-list entries hold z, y and the x-block in 12 + 12 + 8 bits
    G = N.Grains()
    P.dx = 1.0
    L.nx, L.ny, L.nz = 64, 5000, 8
    assert lib.lbdem_psc_near_blocks(C.byref(L), C.byref(P), C.byref(G), 0.25, 8, 8, 8, None) == \
        N.LBDEM_ERR_UNSUPPORTED
    assert b"Ny <= 4096" in lib.lbdem_last_error()


@pytest.mark.skipif(subprocess.run(["which", "gcc"], capture_output=True).returncode != 0, reason="no gcc")
def test_ctypes_descriptors_match_the_header():
    from lbdem_taichi_b200 import _native as N
    structs = {"lbdem_lattice": N.Lattice, "lbdem_grains": N.Grains, "lbdem_psc": N.Psc, "lbdem_dem": N.Dem}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "layout.c")
        exe = os.path.join(tmp, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.check_call(["gcc", "-o", exe, src])
        out = subprocess.check_output([exe], text=True).split("\n")
    got = {}
    for ln in out:
        if ln:
            a, b, c = ln.split()
            got[(a, b)] = int(c)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_binding_raises_with_the_library_message():
    """A non-zero return code becomes LbdemError carrying the function name,
    the code and the library's last error (no device work is attempted: the
    argument checks come first)."""
    from lbdem_taichi_b200 import _native as N
    L = N.Lattice()
    L.nx, L.ny, L.nz = 8, 8, 8
    L.storage, L.omega0, L.scale16 = N.F32, 1.6, 1.0
    L.links, L.status = 8, 8
    with pytest.raises(N.LbdemError) as ei:
        N.call("lbdem_psc_step_f32", C.byref(L), None, None, 0, 0, 1, None)   # src == dst
    msg = str(ei.value)
    assert "lbdem_psc_step_f32" in msg and f"code {N.LBDEM_ERR_ARG}" in msg
    assert "distinct" in msg
    with pytest.raises(N.LbdemError, match="dem: bad descriptor"):
        N.call("lbdem_dem_substeps", None, 1, None)
