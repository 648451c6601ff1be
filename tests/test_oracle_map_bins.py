"""The oracle's binned grains2lattice gives exactly what the reference's
per-cell loop over all grains gives (psclattice3d.py:84-138).

The binned form (``OracleLattice.grains2lattice``) lets the FP64 oracle run the
256^3 and 512x512x256 workloads; ``grains2lattice_all`` is the loop as the
reference writes it.  They must agree bit for bit in owner id, solid fraction
and solid velocity: on the scenarios of every golden fixture that maps grains,
and on random cases with heavy overlap (full covers shadowing partial ones,
equal counts, grains leaving the lattice, grains smaller than a cell, physical
units with an offset domain, non-finite and infinite sizes).
"""
import numpy as np
import pytest

from oracle.oracle import OracleGrains, OracleLattice
from tests.golden_util import load

GOLDENS = ("psc", "hybrid", "coupled", "couette_ladd", "open_x", "open_y", "open_z", "open_xr", "open_exit_x",
           "open_exit_z", "open_yr", "open_zb", "open_slip")


def _both(lat, grains):
    lat.grains2lattice_all(grains)
    ref = (lat.id.copy(), lat.volfrac.copy(), lat.velsolid.copy())
    lat.id[...] = 7
    lat.volfrac[...] = 0.5
    lat.velsolid[...] = 1.0
    lat.grains2lattice(grains)
    return ref, (lat.id, lat.volfrac, lat.velsolid)


def _same(ref, got):
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(got[2], ref[2])


@pytest.mark.parametrize("name", GOLDENS)
def test_binned_map_equals_all_grains_loop_on_goldens(name):
    g = load(name)
    nx, ny, nz = g["ct"].shape
    dom = g["domain"]
    kw = dict(dom_min=(dom[0], dom[2], dom[4]))
    if "dx" in g:
        kw.update(dx=float(g["dx"]), dt=float(g["dt"]), rho_unit=float(g["rho_unit"]))
    lat = OracleLattice(nx, ny, nz, 1.6, psc=True, **kw)
    lat.ct[...] = g["ct"]
    gr = OracleGrains(g["gpos"], g["grad"], g["gvel"], g["gomega"])
    ref, got = _both(lat, gr)
    assert (ref[0] >= 0).sum() > 0
    _same(ref, got)


@pytest.mark.parametrize("seed", range(6))
def test_binned_map_equals_all_grains_loop_random_overlap(seed):
    rng = np.random.default_rng(1000 + seed)
    nx, ny, nz = (int(v) for v in rng.integers(9, 30, 3))
    dx = float(rng.choice([1.0, 0.5, 2e-3]))
    dmin = rng.uniform(-3, 3, 3) * dx
    n = 40
    # centres spread over the box and 2 cells beyond it, radii from below a cell to a third of the box
    pos = dmin + rng.uniform(-2, np.array([nx, ny, nz]) + 2, (n, 3)) * dx
    rad = rng.uniform(0.2, max(nx, ny, nz) / 3, n) * dx
    # exact duplicates and concentric grains: equal counts resolved by id, full covers in the middle of the order
    pos[5] = pos[3]
    rad[5] = rad[3]
    pos[9] = pos[4]
    rad[9] = 0.5 * rad[4]
    # centres on the sub-sample grid (ties on the sphere surface)
    pos[11] = dmin + np.round(pos[11] / dx - dmin / dx, 1) * dx
    vel = rng.normal(0, 1e-3, (n, 3))
    omg = rng.normal(0, 1e-3, (n, 3))
    lat = OracleLattice(nx, ny, nz, 1.6, dx=dx, psc=True, dom_min=tuple(dmin))
    ct = np.ones((nx, ny, nz), np.int32)
    ct[:, :, 0] = 8
    ct[0, :, :] = 32
    lat.ct[...] = ct
    gr = OracleGrains(pos, rad, vel, omg)
    ref, got = _both(lat, gr)
    owners = np.unique(ref[0][ref[0] >= 0])
    assert len(owners) > 10
    assert (ref[1] == 1.0).sum() > 0 and ((ref[1] > 0) & (ref[1] < 1)).sum() > 0
    _same(ref, got)


def test_binned_map_non_finite_and_degenerate_grains():
    nx, ny, nz = 12, 10, 11
    pos = np.array([[5.0, 5.0, 5.0], [np.nan, 4.0, 4.0], [3.0, 3.0, 3.0], [6.0, 2.0, 8.0], [np.inf, 1.0, 1.0],
                    [7.3, 6.1, 4.4], [4.0, 4.0, 4.0]])
    rad = np.array([2.0, 3.0, 0.1, np.nan, 2.0, 0.5, np.inf])
    lat = OracleLattice(nx, ny, nz, 1.6, psc=True)
    gr = OracleGrains(pos, rad, np.zeros((7, 3)), np.zeros((7, 3)))
    ref, got = _both(lat, gr)
    assert (ref[0] == 6).sum() > 0      # the infinite grain covers the cells no earlier grain covers fully
    _same(ref, got)
