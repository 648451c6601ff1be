"""The synthetic dense-suspension case (256^3, 2000 spheres, d ~ U[8, 12],
seeded random sequential addition with a 1 lu gap, velocities N(0, 1e-3),
particle density 2.0) is what its description says, and the same on every
call; the full-size FP64 record starts from exactly these inputs."""
import os

import numpy as np
from scipy.spatial import cKDTree

from lbdem_taichi_b200 import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_dense_suspension_inputs():
    c = cases.case("c2")
    assert c["shape"] == (256, 256, 256)
    pos, rad, vel, mass = cases.particles(c)
    n = c["n"]
    assert n == 2000 and pos.shape == (n, 3) and rad.shape == (n,) and vel.shape == (n, 3)
    assert rad.min() >= 4.0 and rad.max() <= 6.0 and rad.std() > 0.5
    assert (pos >= 0.0).all() and (pos <= 256.0).all()
    # no two spheres closer than their radii plus the 1 lu gap
    pairs = np.array(sorted(cKDTree(pos).query_pairs(2 * 6.0 + 1.0)))
    d = np.linalg.norm(pos[pairs[:, 0]] - pos[pairs[:, 1]], axis=1)
    assert (d >= rad[pairs[:, 0]] + rad[pairs[:, 1]] + 1.0 - 1e-9).all()
    assert abs(vel.std() - 1e-3) < 1e-4 and abs(vel.mean()) < 1e-4
    np.testing.assert_allclose(mass, 2.0 * 4.0 / 3.0 * np.pi * rad ** 3, rtol=1e-15)
    # solid fraction about 6.5 % (E[d^3] = 1040 for d ~ U[8, 12])
    phi = (4.0 / 3.0 * np.pi * rad ** 3).sum() / 256 ** 3
    assert 0.055 < phi < 0.075


def test_workload_is_seeded():
    a = cases.particles(cases.case("c2"))
    b = cases.particles(cases.case("c2"))
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_fp64_records_start_from_the_cases_inputs():
    for name in ("c2", "c1"):
        rec = np.load(os.path.join(GOLDEN, f"{name}_fp64.npz"))
        pos, rad, vel, mass = cases.particles(cases.case(name), int(rec["seed"]))
        np.testing.assert_array_equal(rec["pos0"], pos)
        np.testing.assert_array_equal(rec["rad"], rad)
        np.testing.assert_array_equal(rec["vel0"], vel)
        np.testing.assert_array_equal(rec["mass"], mass)
