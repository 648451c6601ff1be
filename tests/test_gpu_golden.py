"""GPU path vs golden vectors produced by the reference's own source.

Tolerances (FP32 populations stored as deviations f - w, FP32 arithmetic,
against FP64 references):
  populations / density: absolute 1e-6 after three steps
  velocity: max error / max |u| <= 2e-5
  omega (Smagorinsky): absolute 1e-6
  solid fraction / owner id: exact
  particle force and torque: max error / max magnitude <= 1e-4
  DEM state (FP64 on both sides): max error / max magnitude <= 1e-9, contact sets exact
"""
import numpy as np
import pytest

from tests.golden_util import load, relmax

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import lbdem_taichi_b200 as L
    from lbdem_taichi_b200.lbdem.psclattice3d import PSCLattice3D
    from lbdem_taichi_b200.lbm3d.lattice import BasicLattice3D, ForcedLattice3D
    return L, PSCLattice3D, BasicLattice3D, ForcedLattice3D


def _setup(lat, g):
    lat.CT.from_numpy(g["ct"])
    if "rho0" in g:
        lat.rho.from_numpy(g["rho0"])
        lat.vel.from_numpy(g["vel0"])


def test_bgk_smagorinsky(api):
    _, _, Basic, _ = api
    g = load("bgk_smag")
    nx, ny, nz = g["ct"].shape
    lat = Basic(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0)
    _setup(lat, g)
    lat.initialize()
    for s in range(int(g["nsteps"])):
        lat.collide()
        om = lat.omega.to_numpy()
        fl = g["ct"] == 1
        assert np.abs(om - g[f"omega_{s}"])[fl].max() < 1e-6
        lat.stream()
        assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[fl].max() < 1e-6
        assert np.abs(lat.rho.to_numpy() - g[f"rho_{s}"])[fl].max() < 1e-6
        assert relmax(lat.vel.to_numpy()[fl], g[f"vel_{s}"][fl]) < 2e-5
    lat.check_status()


def test_forced(api):
    _, _, _, Forced = api
    g = load("forced")
    nx, ny, nz = g["ct"].shape
    lat = Forced(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, g["force"])
    _setup(lat, g)
    lat.initialize()
    fl = g["ct"] == 1
    for s in range(int(g["nsteps"])):
        lat.collide()
        lat.stream()
        assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[fl].max() < 1e-6
        assert relmax(lat.vel.to_numpy()[fl], g[f"vel_{s}"][fl]) < 2e-5


def _golden_grains_dem(g, dt_dem, rho_p):
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from tests.gpu_util import make_dem
    rad = g["grad"]
    mass = rho_p * 4.0 / 3.0 * np.pi * rad ** 3
    return make_dem(g["domain"], dt_dem, (0, 0, 0), HertzContactConfig(0.3, 0.3, 0.9, 0.9), rad, mass, g["gpos"],
                    g["gvel"], omega=g["gomega"])


def test_psc_physical_units(api):
    _, PSC, _, _ = api
    g = load("psc")
    nx, ny, nz = g["ct"].shape
    dem = _golden_grains_dem(g, float(g["dt"]) / 5, 2500.0)
    lat = PSC(nx, ny, nz, float(g["omega0"]), float(g["dx"]), float(g["dt"]), float(g["rho_unit"]), dem,
              keep_hydroforce=True)
    _setup(lat, g)
    lat.initialize()
    np.testing.assert_array_equal(lat.id.to_numpy(), g["id_init"])
    np.testing.assert_allclose(lat.volfrac.to_numpy(), g["volfrac_init"], rtol=0, atol=1e-7)
    assert relmax(lat.velsolid.to_numpy(), g["velsolid_init"]) < 1e-5
    fl = g["ct"] == 1
    for s in range(int(g["nsteps"])):
        lat.collide()
        np.testing.assert_array_equal(lat.id.to_numpy(), g[f"id_{s}"])
        assert np.abs(lat.weight.to_numpy() - g[f"weight_{s}"]).max() < 1e-6
        assert relmax(lat.hydroforce.to_numpy(), g[f"hydroforce_{s}"]) < 1e-4
        assert relmax(dem.gf.force_fluid.to_numpy(), g[f"force_fluid_{s}"]) < 1e-4
        assert relmax(dem.gf.moment_fluid.to_numpy(), g[f"moment_fluid_{s}"]) < 1e-4
        lat.stream()
        assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[fl].max() < 1e-6
        assert relmax(lat.vel.to_numpy()[fl], g[f"vel_{s}"][fl]) < 2e-5
    lat.check_status()


@pytest.mark.parametrize("read_every_step", [True, False])
def test_moving_walls_ladd(api, read_every_step):
    """VEL_LADD walls (lbm_solver3d.py:222-225) around a PSC sphere.  Reading
    the fields after every step streams through lbdem_stream_moments; reading
    only at the end streams inside the fused step kernel."""
    _, PSC, _, _ = api
    g = load("couette_ladd")
    nx, ny, nz = g["ct"].shape
    dem = _golden_grains_dem(g, 0.25, 2.0)
    lat = PSC(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem, stress=True)
    _setup(lat, g)
    lat.initialize()
    fl = g["ct"] == 1
    n = int(g["nsteps"])
    for s in range(n):
        lat.collide()
        assert relmax(dem.gf.force_fluid.to_numpy(), g[f"force_fluid_{s}"]) < 1e-4
        assert relmax(dem.gf.moment_fluid.to_numpy(), g[f"moment_fluid_{s}"]) < 1e-4
        lat.stream()
        if read_every_step or s == n - 1:
            assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[fl].max() < 1e-6
            assert np.abs(lat.rho.to_numpy() - g[f"rho_{s}"])[fl].max() < 1e-6
            assert relmax(lat.vel.to_numpy()[fl], g[f"vel_{s}"][fl]) < 2e-5
            # stress diagnostics of the shear driver (lbm_solver3d.py:347-456)
            lat.compute_stress()
            for k in ("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz",
                      "shear_stress_mag"):
                assert np.abs(getattr(lat, k).to_numpy() - g[f"{k}_{s}"])[fl].max() < 2e-7, k
            for key, (axis, pos) in (("plane_top", (2, nz - 2)), ("plane_y", (1, 3)), ("plane_x", (0, 4))):
                assert np.abs(lat.compute_plane_average_stress(axis, pos) - g[f"{key}_{s}"]).max() < 2e-7, key
    lat.check_status()


@pytest.mark.parametrize("storage,tol", [("f32", 2e-7), ("f16", 5e-5), ("bf16", 5e-4)])
def test_stress_fused_into_the_step(api, monkeypatch, storage, tol):
    """The shear driver's loop (shear_fullyresolved.py:226-233): compute_stress()
    after every stream.  The next collide() gathers exactly the state the call
    refers to and writes the stress as an optional output of the fused step;
    no separate stress pass runs.  The fields read after that collide equal the
    reference's stress of the previous step (stresses up to 1.2e-3 here):
    FP32 storage within 2e-7; the 16-bit forms within the rounding of their
    stored populations, 5e-5 (FP16) and 5e-4 (BF16)."""
    from lbdem_taichi_b200 import _native as N
    _, PSC, _, _ = api
    g = load("couette_ladd")
    nx, ny, nz = g["ct"].shape
    dem = _golden_grains_dem(g, 0.25, 2.0)
    lat = PSC(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem, stress=True, storage=storage)
    _setup(lat, g)
    lat.initialize()
    fl = g["ct"] == 1
    calls = []
    orig = N.call
    monkeypatch.setattr(N, "call", lambda name, *a: (calls.append(name), orig(name, *a))[1])
    names = ("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz", "shear_stress_mag")
    checked = 0
    for s in range(int(g["nsteps"])):
        lat.collide()
        if s > 0:
            for k in names:
                assert np.abs(getattr(lat, k).to_numpy() - g[f"{k}_{s - 1}"])[fl].max() < tol, (k, s)
            for key, (axis, pos) in (("plane_top", (2, nz - 2)), ("plane_y", (1, 3)), ("plane_x", (0, 4))):
                got = lat.compute_plane_average_stress(axis, pos)
                assert np.abs(got - g[f"{key}_{s - 1}"]).max() < tol, key
            checked += 1
        lat.stream()
        lat.compute_stress()
    assert checked >= 2
    assert "lbdem_stress" not in calls
    # a read with a compute_stress() pending evaluates it in a pass of its own: the last step's stress
    for k in names:
        assert np.abs(getattr(lat, k).to_numpy() - g[f"{k}_{s}"])[fl].max() < tol, k
    assert calls.count("lbdem_stress") == 1
    lat.check_status()


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_stress_fused_equals_separate_pass(api, storage):
    """The stress the fused step writes equals the separate pass's
    (lbdem_stress) on the same stored state, for every storage form: the same
    FP32 arithmetic in another order (within 1e-6 of the largest value)."""
    _, PSC, _, _ = api
    g = load("couette_ladd")
    nx, ny, nz = g["ct"].shape
    dem = _golden_grains_dem(g, 0.25, 2.0)
    lat = PSC(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem, stress=True, storage=storage)
    _setup(lat, g)
    lat.initialize()
    fl = g["ct"] == 1
    names = ("stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz", "shear_stress_mag")
    for s in range(int(g["nsteps"])):
        lat.collide()
        lat.stream()
        lat.compute_stress()
        sep = [getattr(lat, k).to_numpy() for k in names]       # read with the call pending: separate pass
        lat.compute_stress()                                      # pending again: fused into the next collide
        lat.collide()
        fused = [getattr(lat, k).to_numpy() for k in names]
        for k, a, b in zip(names, sep, fused):
            assert np.abs(a - b)[fl].max() <= 1e-6 * max(np.abs(a[fl]).max(), 1e-30), (k, s)
        lat.stream()
    lat.check_status()


def test_hybrid_psc_smagorinsky(api):
    _, PSC, _, _ = api
    g = load("hybrid")
    nx, ny, nz = g["ct"].shape
    dem = _golden_grains_dem(g, 0.1, 2.5)
    lat = PSC(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem, smagorinsky="reference", skip_inlet=True,
              keep_hydroforce=True)
    _setup(lat, g)
    lat.initialize()
    fl = g["ct"] == 1
    for s in range(int(g["nsteps"])):
        lat.collide()
        np.testing.assert_array_equal(lat.id.to_numpy(), g[f"id_{s}"])
        assert np.abs(lat.omega.to_numpy() - g[f"omega_{s}"])[fl].max() < 1e-6
        assert np.abs(lat.weight.to_numpy() - g[f"weight_{s}"]).max() < 1e-6
        assert relmax(dem.gf.force_fluid.to_numpy(), g[f"force_fluid_{s}"]) < 1e-4
        assert relmax(dem.gf.moment_fluid.to_numpy(), g[f"moment_fluid_{s}"]) < 1e-4
        lat.stream()
        assert np.abs(lat.f.to_numpy() - g[f"f_{s}"])[fl].max() < 1e-6


@pytest.mark.parametrize("model", ["hertz", "linear"])
def test_dem_golden(model):
    from tests.gpu_util import golden_dem
    g = load(f"dem_{model}")
    dem = golden_dem(g, model)
    dem.gf.force_fluid.from_numpy(g["force_fluid"])
    dem.gf.moment_fluid.from_numpy(g["moment_fluid"])
    for s in range(1, int(g["nsub"]) + 1):
        dem.run_simulation()
        if s % 5:
            continue
        for k in ("position", "velocity", "omega", "quaternion", "force", "moment", "acceleration", "omega_dot"):
            assert relmax(getattr(dem.gf, k).to_numpy(), g[f"{k}_{s}"]) < 1e-9, (k, s)
        con = dem.active_contacts()
        ref = {(int(a), int(b)): sh for (a, b), sh in zip(g[f"pairs_{s}"], g[f"shear_{s}"])}
        assert set(con) == set(ref), s
        for k, sh in ref.items():
            assert np.allclose(con[k][2], sh, rtol=1e-8, atol=1e-12)
        np.testing.assert_array_equal(dem.wcf_active.cpu().numpy().astype(bool), g[f"wact_{s}"])
    dem.check_status()


def test_coupled_loop(api):
    _, PSC, _, _ = api
    from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig
    from tests.gpu_util import make_dem
    g = load("coupled")
    nx, ny, nz = g["ct"].shape
    rad = g["grad"]
    mass = float(g["density"]) * 4.0 / 3.0 * np.pi * rad ** 3
    dem = make_dem(g["domain"], float(g["dt_dem"]), g["gravity"], HertzContactConfig(0.3, 0.3, 0.9, 0.9), rad, mass,
                   g["gpos"], g["gvel"], omega=g["gomega"], periodic=(True, True, False))
    lat = PSC(nx, ny, nz, float(g["omega0"]), 1.0, 1.0, 1.0, dem)
    lat.CT.from_numpy(g["ct"])
    lat.initialize()
    fl = g["ct"] == 1
    for s in range(int(g["nsteps"])):
        lat.step(int(g["sub"]))
        np.testing.assert_array_equal(lat.id.to_numpy(), g[f"id_{s}"])
        for k in ("position", "velocity", "omega"):
            assert relmax(getattr(dem.gf, k).to_numpy(), g[f"{k}_{s}"]) < 1e-7, (k, s)
        for k in ("force_fluid", "moment_fluid"):
            assert relmax(getattr(dem.gf, k).to_numpy(), g[f"{k}_{s}"]) < 1e-4, (k, s)
        assert relmax(lat.vel.to_numpy()[fl], g[f"vel_{s}"][fl]) < 2e-5
    assert np.abs(lat.f.to_numpy() - g["f_last"])[fl].max() < 1e-6
    lat.check_status()
    dem.check_status()
