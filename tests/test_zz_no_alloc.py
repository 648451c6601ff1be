"""The allocation-free conservation sums (lbdem_global_sums_f64_noalloc).

Some callers own the lattice buffers but cannot allocate device memory: a
host that reaches the library only through its C ABI with buffers lent by
another component, or a process whose GPU memory is fully reserved by a
framework's caching allocator.  They cannot hand lbdem_global_sums_f64 its
scratch, so this entry point keeps the block partials in a library-owned
64 KB device array instead (lattices of at most 2^26 cells).

The GPU test calls both entry points through the C ABI on two calls in a row
and holds them to each other (FP64; different block counts, so a different
summation order: relative tolerance 1e-12) and to an FP64 sum on the host of
the same buffer, decoded there from its stored values, over the updated
cells (the device sums each cell's 19 deviations in FP32: relative 1e-9 on the
mass, 1e-7 of the mass on the momentum components).
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
    lat.vel.from_numpy(0.02 * rng.uniform(-1, 1, (nx, ny, nz, 3)) + np.array([0.01, -0.004, 0.0]))
    lat.rho.from_numpy(1.0 + 0.01 * rng.uniform(-1, 1, (nx, ny, nz)))
    lat.initialize()
    for _ in range(3):
        lat.collide()
        lat.stream()
    return lat, ct


def _host_sums(lat, buf, ct):
    """FP64 [mass, momentum] of the updated cells of population buffer `buf`."""
    from lbdem_taichi_b200.lbm3d.lattice import C_Q, W
    d = lat._unblock(lat._f[buf], 19) * (np.asarray(W)[:, None] / lat._scale)   # f - w, (19, Ncells)
    keep = (ct != 8).transpose(2, 1, 0).reshape(-1)                               # z, y, x cell order
    d = d[:, keep]
    c = np.asarray(C_Q, np.float64)
    return np.array([keep.sum() + d.sum(), *(c.T @ d).sum(axis=1)])


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_noalloc_sums_match_scratch_sums(storage):
    import torch
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    lat, ct = _lattice(storage)
    lat._sync_inputs()
    buf = lat._cur
    stream = torch.cuda.current_stream().cuda_stream
    ref_out = torch.zeros(4, dtype=torch.float64, device="cuda")
    partials = torch.zeros(N.SUM_PARTIALS, dtype=torch.float64, device="cuda")
    rc = lib.lbdem_global_sums_f64(C.byref(lat._lat), buf, ref_out.data_ptr(), partials.data_ptr(), stream)
    assert rc == 0, lib.lbdem_last_error()
    ref = ref_out.cpu().numpy()
    host = _host_sums(lat, buf, ct)
    mass = host[0]
    assert mass > 0.9 * lat.Nx * lat.Ny * (lat.Nz - 2)
    assert np.abs(host[1:]).max() > 1.0      # a net momentum to compare, not only round-off
    np.testing.assert_allclose(ref[0], mass, rtol=1e-9)
    np.testing.assert_allclose(ref[1:], host[1:], rtol=0, atol=1e-7 * mass)
    for _ in range(2):
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.lbdem_global_sums_f64_noalloc(C.byref(lat._lat), buf, out.data_ptr(), stream)
        assert rc == 0, lib.lbdem_last_error()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * abs(ref[0]))
        np.testing.assert_allclose(got[0], mass, rtol=1e-9)
        np.testing.assert_allclose(got[1:], host[1:], rtol=0, atol=1e-7 * mass)


def test_noalloc_sums_reject_lattices_beyond_the_static_scratch():
    """More than 2^26 cells (but within the 32-bit offset limit of the other
    entry points): refused on the host by the allocation-free check itself,
    before any device work."""
    from lbdem_taichi_b200 import _native as N
    lib = N.load()
    L = N.Lattice()
    L.nx, L.ny, L.nz = 1024, 1024, 65         # 68.2 M cells, 1.3e9 population elements < 2^32
    L.storage = N.F32
    L.omega0 = 1.6
    L.scale16 = 1.0
    L.links, L.status = 8, 8      # never dereferenced: the size check comes first
    rc = lib.lbdem_global_sums_f64_noalloc(C.byref(L), 0, 8, None)
    assert rc == N.LBDEM_ERR_ARG
    assert b"allocation-free sums cover at most 67108864 cells" in lib.lbdem_last_error()
