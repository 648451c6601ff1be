"""The allocation-free conservation sums (lbdem_global_sums_f64_noalloc).

Some callers own the lattice buffers but cannot allocate device memory: a
host that reaches the library only through its C ABI with buffers lent by
another component, or a process whose GPU memory is fully reserved by a
framework's caching allocator.  They cannot hand lbdem_global_sums_f64 its
scratch, so this entry point keeps the block partials in a library-owned
device array instead.  These tests call both entry points through the C ABI
and require the same totals (FP64; the two use different block counts, so
the summation order differs: relative tolerance 1e-12) on two calls in a row.
"""
import ctypes as C

import numpy as np
import pytest


def _lattice(storage):
    from lbdem_taichi_b200.lbm3d.lattice import BasicLattice3D
    rng = np.random.default_rng(31)
    nx, ny, nz = 64, 40, 36
    lat = BasicLattice3D(nx, ny, nz, 1 / 0.6, 1.0, 1.0, 1.0, storage=storage)
    ct = np.ones((nx, ny, nz), np.int32)
    ct[:, :, 0] = ct[:, :, -1] = 8
    lat.CT.from_numpy(ct)
    lat.vel.from_numpy(0.02 * rng.uniform(-1, 1, (nx, ny, nz, 3)))
    lat.rho.from_numpy(1.0 + 0.01 * rng.uniform(-1, 1, (nx, ny, nz)))
    lat.initialize()
    for _ in range(3):
        lat.collide()
        lat.stream()
    return lat


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_noalloc_sums_match_scratch_sums(storage):
    import torch
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    lat = _lattice(storage)
    lat._sync_inputs()
    buf = lat._cur
    stream = torch.cuda.current_stream().cuda_stream
    ref_out = torch.zeros(4, dtype=torch.float64, device="cuda")
    partials = torch.zeros(N.SUM_PARTIALS, dtype=torch.float64, device="cuda")
    rc = lib.lbdem_global_sums_f64(C.byref(lat._lat), buf, ref_out.data_ptr(), partials.data_ptr(), stream)
    assert rc == 0, lib.lbdem_last_error()
    ref = ref_out.cpu().numpy()
    assert ref[0] > 0.9 * lat.Nx * lat.Ny * (lat.Nz - 2)
    for _ in range(2):
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.lbdem_global_sums_f64_noalloc(C.byref(lat._lat), buf, out.data_ptr(), stream)
        assert rc == 0, lib.lbdem_last_error()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * abs(ref[0]))


def test_noalloc_sums_reject_lattices_beyond_the_static_scratch():
    """More than 2^28 cells: refused on the host, before any device work."""
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    L = N.Lattice()
    L.nx, L.ny, L.nz = 1024, 1024, 257
    L.storage = N.F32
    L.omega0 = 1.6
    L.scale16 = 1.0
    L.links, L.status = 8, 8      # never dereferenced: the size check comes first
    rc = lib.lbdem_global_sums_f64_noalloc(C.byref(L), 0, 8, None)
    assert rc == N.LBDEM_ERR_ARG
    assert b"at most" in lib.lbdem_last_error()
