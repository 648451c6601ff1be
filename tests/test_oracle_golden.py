"""Pin the FP64 C oracle against golden vectors produced by running the
reference's own Python source (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle.oracle import OracleDEM, OracleGrains, OracleLattice, bpcd_table_size
from tests.golden_util import dem_params, load, relmax

TOL = 1e-11   # FP64 vs FP64 (different summation order in a few places)


def _lattice_from(g, **kw):
    nx, ny, nz = g["ct"].shape
    lat = OracleLattice(nx, ny, nz, float(g["omega0"]), **kw)
    lat.ct[...] = g["ct"]
    if "rho0" in g:
        lat.rho[...] = g["rho0"]
        lat.vel[...] = g["vel0"]
    return lat


def test_bgk_smagorinsky_matches_reference():
    g = load("bgk_smag")
    lat = _lattice_from(g, smag=True, smag_cs=float(g["cs"]), skip_inlet=True)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.collide()
        assert relmax(lat.omega, g[f"omega_{s}"]) < TOL
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.rho, g[f"rho_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL
    # Smagorinsky actually changed omega
    assert g["omega_2"].min() < float(g["omega0"]) - 1e-3


def test_forced_matches_reference():
    g = load("forced")
    lat = _lattice_from(g, force=g["force"])
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.collide()
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL


def _grains(g):
    return OracleGrains(g["gpos"], g["grad"], g["gvel"], g["gomega"])


def test_psc_matches_reference():
    g = load("psc")
    dom = g["domain"]
    lat = _lattice_from(g, psc=True, dx=float(g["dx"]), dt=float(g["dt"]), rho_unit=float(g["rho_unit"]),
                        dom_min=(dom[0], dom[2], dom[4]))
    gr = _grains(g)
    lat.initialize()
    lat.grains2lattice(gr)
    np.testing.assert_array_equal(lat.id, g["id_init"])
    np.testing.assert_array_equal(lat.volfrac, g["volfrac_init"])
    assert relmax(lat.velsolid, g["velsolid_init"]) < TOL
    for s in range(int(g["nsteps"])):
        lat.grains2lattice(gr)
        lat.collide()
        lat.lattice2grains(gr)
        np.testing.assert_array_equal(lat.id, g[f"id_{s}"])
        np.testing.assert_array_equal(lat.volfrac, g[f"volfrac_{s}"])
        assert relmax(lat.weight, g[f"weight_{s}"]) < TOL
        assert relmax(lat.hydroforce, g[f"hydroforce_{s}"]) < TOL
        assert relmax(gr.force_fluid, g[f"force_fluid_{s}"]) < TOL
        assert relmax(gr.moment_fluid, g[f"moment_fluid_{s}"]) < TOL
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL


def test_moving_walls_ladd_match_reference():
    """VEL_LADD walls (modified bounce-back with the wall velocity,
    lbm_solver3d.py:222-225) around a PSC sphere."""
    g = load("couette_ladd")
    dom = g["domain"]
    lat = _lattice_from(g, psc=True, dom_min=(dom[0], dom[2], dom[4]))
    gr = _grains(g)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.grains2lattice(gr)
        lat.collide()
        lat.lattice2grains(gr)
        assert relmax(gr.force_fluid, g[f"force_fluid_{s}"]) < TOL
        assert relmax(gr.moment_fluid, g[f"moment_fluid_{s}"]) < TOL
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.rho, g[f"rho_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL
        st = lat.compute_stress()
        for m, k in enumerate(("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz",
                               "shear_stress_mag")):
            assert relmax(st[..., m], g[f"{k}_{s}"]) < 1e-9, k
        nz = lat.shape[2]
        for key, (axis, pos) in (("plane_top", (2, nz - 2)), ("plane_y", (1, 3)), ("plane_x", (0, 4))):
            assert relmax(lat.plane_average_stress(axis, pos), g[f"{key}_{s}"]) < 1e-9, key
    # the walls drive a shear: the wall-adjacent fluid moves with them
    assert g["vel_2"][:, :, -2, 0].mean() > 0 > g["vel_2"][:, :, 1, 0].mean()


OPEN_SCENARIOS = ("open_x", "open_y", "open_z", "open_xr", "open_exit_x", "open_exit_z", "open_yr", "open_zb",
                  "open_slip")


@pytest.mark.parametrize("name", OPEN_SCENARIOS)
def test_open_boundaries_match_reference(name):
    """Wet-node boundaries of the second stream pass (lbm_solver3d.py:242-250):
    Zou-He velocity / pressure on all six faces, convective exits and Ladd
    velocity inlets (with the inlet neighbour rule, :225-229), around a PSC
    sphere."""
    g = load(name)
    dom = g["domain"]
    lat = _lattice_from(g, psc=True, dom_min=(dom[0], dom[2], dom[4]))
    gr = _grains(g)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.grains2lattice(gr)
        lat.collide()
        lat.lattice2grains(gr)
        assert relmax(gr.force_fluid, g[f"force_fluid_{s}"]) < TOL
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.rho, g[f"rho_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL
    # the boundaries act: the flow through the lattice is along the open axis
    axis = int(np.argmax(g["ct"].shape))
    assert abs(g["vel_3"][..., axis].mean()) > 1e-3


def test_open_boundaries_smagorinsky_match_reference():
    """BasicLattice3D (Smagorinsky; initialize/collide skip the Ladd inlet) with
    a Ladd inlet, a convective exit and free-slip walls."""
    g = load("open_smag")
    lat = _lattice_from(g, smag=True, smag_cs=float(g["cs"]), skip_inlet=True)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.collide()
        assert relmax(lat.omega, g[f"omega_{s}"]) < TOL
        lat.stream()
        assert relmax(lat.f, g[f"f_{s}"]) < TOL
        assert relmax(lat.rho, g[f"rho_{s}"]) < TOL
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL
    assert g["omega_3"].min() < float(g["omega0"]) - 1e-3


def test_hybrid_psc_smagorinsky_matches_reference():
    g = load("hybrid")
    dom = g["domain"]
    lat = _lattice_from(g, psc=True, smag=True, smag_cs=float(g["cs"]), skip_inlet=True,
                        dom_min=(dom[0], dom[2], dom[4]))
    gr = _grains(g)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.grains2lattice(gr)
        lat.collide()
        np.testing.assert_array_equal(lat.id, g[f"id_{s}"])
        assert relmax(lat.omega, g[f"omega_{s}"]) < TOL
        assert relmax(lat.weight, g[f"weight_{s}"]) < TOL
        assert relmax(lat.hydroforce, g[f"hydroforce_{s}"]) < TOL
        lat.stream()
        lat.lattice2grains(gr)
        assert relmax(gr.force_fluid, g[f"force_fluid_{s}"]) < TOL
        assert relmax(gr.moment_fluid, g[f"moment_fluid_{s}"]) < TOL
        assert relmax(lat.f, g[f"f_{s}"]) < TOL


@pytest.mark.parametrize("model", ["hertz", "linear"])
def test_dem_matches_reference(model):
    g = load(f"dem_{model}")
    d = OracleDEM(g["gpos"], g["gvel"], g["grad"], g["mass"], **dem_params(g, model))
    assert d.d.table_size == int(g["table_size"])
    assert abs(d.d.cell_size - float(g["cell_size"])) < 1e-12
    d.force_fluid[...] = g["force_fluid"]
    d.moment_fluid[...] = g["moment_fluid"]
    for s in range(1, int(g["nsub"]) + 1):
        d.run_simulation()
        assert d.status == 0
        if s % 5:
            continue
        for k, mine in (("position", d.pos), ("velocity", d.vel), ("omega", d.omega),
                        ("quaternion", d.quat), ("force", d.force), ("moment", d.moment),
                        ("acceleration", d.acc), ("omega_dot", d.omega_dot)):
            assert relmax(mine, g[f"{k}_{s}"]) < 1e-9, (k, s)
        pairs = d.active_pairs()
        ref = {(int(a), int(b)): sh for (a, b), sh in zip(g[f"pairs_{s}"], g[f"shear_{s}"])}
        assert set(pairs) == set(ref), s
        for k in ref:
            assert np.allclose(pairs[k], ref[k], rtol=1e-8, atol=1e-12)
        np.testing.assert_array_equal(d.wcf_active.astype(bool), g[f"wact_{s}"])
        assert relmax(d.wcf_shear, g[f"wshear_{s}"], floor=1e-12) < 1e-8


def test_coupled_driver_loop_matches_reference():
    g = load("coupled")
    dom = g["domain"]
    nx, ny, nz = g["ct"].shape
    lat = OracleLattice(nx, ny, nz, float(g["omega0"]), psc=True, dom_min=(dom[0], dom[2], dom[4]))
    lat.ct[...] = g["ct"]
    rad = g["grad"]
    mass = float(g["density"]) * 4.0 / 3.0 * np.pi * rad ** 3
    d = OracleDEM(g["gpos"], g["gvel"], rad, mass, dt=float(g["dt_dem"]), gravity=g["gravity"], domain=dom,
                  periodic=(True, True, False), model="hertz", E=1e5, nu=0.3, wall_E=1e5, wall_nu=0.3,
                  pp_mu=0.3, pw_mu=0.3, pp_e=0.9, pw_e=0.9, max_coord=16, omega=g["gomega"])
    gr = OracleGrains(d.pos, d.radius, d.vel, d.omega)
    # share DEM state arrays with the coupling view
    gr.pos, gr.vel, gr.omega = d.pos, d.vel, d.omega
    gr.force_fluid, gr.moment_fluid = d.force_fluid, d.moment_fluid
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.grains2lattice(gr)
        lat.collide()
        lat.lattice2grains(gr)
        lat.stream()
        for _ in range(int(g["sub"])):
            d.run_simulation()
        np.testing.assert_array_equal(lat.id, g[f"id_{s}"])
        for k, mine in (("position", d.pos), ("velocity", d.vel), ("force_fluid", d.force_fluid),
                        ("moment_fluid", d.moment_fluid), ("omega", d.omega)):
            assert relmax(mine, g[f"{k}_{s}"]) < 1e-9, (k, s)
        assert relmax(lat.vel, g[f"vel_{s}"]) < TOL
    assert relmax(lat.f, g["f_last"]) < TOL


def test_table_size_rule():
    # bpcd.py:48-65: clamp to [2^20, 2^22]
    assert bpcd_table_size(10, 1.0, (0, 0, 0), (4, 4, 4)) == 1 << 20
    assert bpcd_table_size(10, 0.01, (0, 0, 0), (100, 100, 100)) == 1 << 22
