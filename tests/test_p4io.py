"""p4p / p4c files against the reference's own DEMSolver.save_single output
(tests/golden/p4io.npz, made by tests/golden/make_golden.py from the
reference's source): the writers reproduce its text byte for byte from the
same arrays, and the reader parses it back (values to the 7 significant
digits the format keeps)."""
import io

import numpy as np

from lbdem_taichi_b200.dem3d.p4io import read_p4p, write_p4c, write_p4p
from tests.golden_util import load


def test_p4p_frame_matches_the_reference_text():
    g = load("p4io")
    buf = io.StringIO()
    write_p4p(buf, float(g["t"]), g["ID"], g["group"], g["radius"], g["mass"], g["position"], g["velocity"])
    assert buf.getvalue() == str(g["p4p"])


def test_p4c_frame_matches_the_reference_text():
    g = load("p4io")
    ID = g["ID"]
    rows = [[ID[i], ID[j], *p, *f] for i, j, p, f in zip(g["ci"], g["cj"], g["cpos"], g["cforce"])]
    assert len(rows) >= 2
    buf = io.StringIO()
    write_p4c(buf, float(g["t"]), rows)       # the reference's slot order
    assert buf.getvalue() == str(g["p4c"])
    # DEMSolver.save_single orders the rows by (P1, P2): the same lines
    buf = io.StringIO()
    write_p4c(buf, float(g["t"]), sorted(rows, key=lambda r: (r[0], r[1])))
    ours, ref = buf.getvalue().splitlines(), str(g["p4c"]).splitlines()
    assert ours[:3] == ref[:3] and sorted(ours[3:]) == sorted(ref[3:])


def test_empty_contact_frame():
    buf = io.StringIO()
    write_p4c(buf, 0.5, [])
    assert buf.getvalue() == "TIMESTEP  CONTACTS\n0.5 0\nP1  P2  CX  CY  CZ  FX  FY  FZ\n"


def test_reader_parses_the_reference_frame(tmp_path):
    g = load("p4io")
    path = tmp_path / "frame.p4p"
    path.write_text(str(g["p4p"]))
    p = read_p4p(str(path))
    np.testing.assert_array_equal(p["ID"], g["ID"])
    np.testing.assert_array_equal(p["group"], g["group"])
    for k, ref in (("radius", g["radius"]), ("mass", g["mass"]), ("pos", g["position"]), ("vel", g["velocity"])):
        np.testing.assert_allclose(p[k], ref, rtol=6e-7, atol=0, err_msg=k)
    r, m = p["radius"][-1], p["mass"][-1]
    assert p["density"] == 3 * m / (4 * np.pi * r ** 3)


def test_reader_takes_rows_in_any_id_order(tmp_path):
    path = tmp_path / "shuffled.p4p"
    path.write_text("TIMESTEP  PARTICLES\n0 2\nID  GROUP  RAD  MASS  PX  PY  PZ  VX  VY  VZ\n"
                    "2 1 1.5 3.0 4 5 6 0.1 0.2 0.3\n1 0 2.5 7.0 1 2 3 -0.1 -0.2 -0.3\n")
    p = read_p4p(str(path))
    np.testing.assert_array_equal(p["ID"], [1, 2])
    np.testing.assert_array_equal(p["group"], [0, 1])
    np.testing.assert_array_equal(p["pos"], [[1, 2, 3], [4, 5, 6]])
    np.testing.assert_array_equal(p["vel"], [[-0.1, -0.2, -0.3], [0.1, 0.2, 0.3]])


class _Field:
    def __init__(self, a):
        self._a = np.asarray(a)

    def to_numpy(self):
        return self._a.copy()


def test_demsolver_save_single_writes_the_reference_frame(capsys):
    """DEMSolver.save_single on a stand-in for the device state (the golden's
    arrays and active contacts): the reference's p4p text, and its p4c lines
    in (P1, P2) order."""
    from types import SimpleNamespace
    from lbdem_taichi_b200.dem3d.demsolver import DEMSolver
    g = load("p4io")
    dem = object.__new__(DEMSolver)
    dem.n = len(g["ID"])
    dem.gf = SimpleNamespace(ID=_Field(g["ID"]), groupID=_Field(g["group"]), radius=_Field(g["radius"]),
                             mass=_Field(g["mass"]), position=_Field(g["position"]), velocity=_Field(g["velocity"]))
    con = {(int(i), int(j)): (p, f, np.zeros(3)) for i, j, p, f in zip(g["ci"], g["cj"], g["cpos"], g["cforce"])}
    dem.active_contacts = lambda: con
    p4p, p4c = io.StringIO(), io.StringIO()
    dem.save_single(p4p, p4c, float(g["t"]))
    assert p4p.getvalue() == str(g["p4p"])
    ours, ref = p4c.getvalue().splitlines(), str(g["p4c"]).splitlines()
    assert ours[:3] == ref[:3] and sorted(ours[3:]) == sorted(ref[3:])
    assert ours[3:] == sorted(ours[3:], key=lambda ln: tuple(int(v) for v in ln.split()[:2]))


def test_demsolver_init_particle_fields_reads_the_file(tmp_path, monkeypatch):
    """DEMSolver.init_particle_fields hands the parsed file to the device
    allocation (stood in for here): IDs, groups, radii, masses, positions,
    velocities and the density, with the domain bounds."""
    from lbdem_taichi_b200 import _native
    from lbdem_taichi_b200.dem3d.demsolver import DEMSolver
    g = load("p4io")
    path = tmp_path / "frame.p4p"
    path.write_text(str(g["p4p"]))
    got = {}
    monkeypatch.setattr(_native, "require_cuda", lambda: None)
    dem = object.__new__(DEMSolver)
    dem._allocate = lambda *a: got.setdefault("args", a)
    dem.init_particle_fields(str(path), (0.0, 0.0, 0.0), (40.0, 30.0, 30.0))
    ID, group, radius, mass, pos, vel, density, dmin, dmax = got["args"]
    np.testing.assert_array_equal(ID, g["ID"])
    np.testing.assert_array_equal(group, g["group"])
    np.testing.assert_allclose(radius, g["radius"], rtol=6e-7)
    np.testing.assert_allclose(pos, g["position"], rtol=6e-7)
    np.testing.assert_allclose(vel, g["velocity"], rtol=6e-7)
    assert density == 3 * mass[-1] / (4 * np.pi * radius[-1] ** 3)
    assert dmin == (0.0, 0.0, 0.0) and dmax == (40.0, 30.0, 30.0)
