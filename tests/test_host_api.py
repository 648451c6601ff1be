"""Host-side helpers that drivers call, against the reference's own code
(tests/golden/host_api.npz, made by tests/golden/make_golden.py under the
NumPy Taichi shim): UnitConverter conversions, DEMSolverConfig state after
its setters (walls, periodic flags, extended bounds, material properties,
contact-model updates), summary() text for both contact models, and the
inputs that raise ValueError."""
import numpy as np
import pytest

from tests.golden_util import load


def _cfgs():
    from lbdem_taichi_b200 import Vector3
    from lbdem_taichi_b200.dem3d.demconfig import (DEMSolverConfig, DomainBounds, HertzContactConfig,
                                                   LinearContactConfig)
    cfg = DEMSolverConfig(domain=DomainBounds(0.0, 1.0, 0.0, 2.0, -1.0, 3.0), dt=1e-4,
                          gravity=Vector3(0.0, 0.0, -9.81),
                          contact_model=HertzContactConfig(pp_friction=0.3, pw_friction=0.4, pp_restitution=0.9,
                                                           pw_restitution=0.8))
    cfg.set_particle_properties(elastic_modulus=1e6, poisson_ratio=0.25, density=2650.0, max_coordinate_number=12)
    cfg.set_wall_properties(density=2500.0, elastic_modulus=2e6, poisson_ratio=0.3)
    cfg.set_periodic_boundaries(True, False, True)
    cfg.update_contact_model(pp_friction=0.5)
    lin = DEMSolverConfig(domain=DomainBounds(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), dt=2e-4, gravity=Vector3(0.0, -1.0, 0.0),
                          contact_model=LinearContactConfig(stiffness_normal=1e5, stiffness_tangential=5e4,
                                                            damping_normal=0.1, damping_tangential=0.05,
                                                            pp_friction=0.2, pw_friction=0.3))
    return cfg, lin


def test_unit_converter():
    from lbdem_taichi_b200.lbm3d.lbmutils import UnitConverter
    g = load("host_api")
    uc = UnitConverter(2e-3, 1e-4, 1000.0)
    for name, ref in zip(g["conv_names"], g["conv"]):
        got = [getattr(uc, str(name))(v) for v in (0.5, 3.0)]
        np.testing.assert_array_equal(got, ref, err_msg=str(name))


def test_config_state_after_setters():
    g = load("host_api")
    cfg, _ = _cfgs()
    np.testing.assert_array_equal(cfg.boundaryType, g["boundary_type"])
    np.testing.assert_array_equal(np.asarray(cfg.wall_distances, float), g["wall_distances"])
    np.testing.assert_array_equal(np.array([np.asarray(v, float) for v in cfg.wall_normals]), g["wall_normals"])
    np.testing.assert_array_equal(np.asarray(cfg.domain_min, float), g["domain_min"])
    np.testing.assert_array_equal(np.asarray(cfg.domain_max, float), g["domain_max"])
    pp, wp = cfg.particle_props, cfg.wall_props
    np.testing.assert_array_equal([pp.elastic_modulus, pp.poisson_ratio, pp.density, pp.max_coordinate_number],
                                  g["particle_props"])
    np.testing.assert_array_equal([wp.density, wp.elastic_modulus, wp.poisson_ratio], g["wall_props"])
    assert cfg.contact_model.pp_friction == g["pp_friction"]


def test_summary_text():
    g = load("host_api")
    cfg, lin = _cfgs()
    assert cfg.summary() == str(g["summary_hertz"])
    assert lin.summary() == str(g["summary_linear"])


def test_invalid_inputs_raise_as_the_reference():
    from lbdem_taichi_b200 import Vector3
    from lbdem_taichi_b200.dem3d.demconfig import (DEMSolverConfig, DomainBounds, HertzContactConfig,
                                                   LinearContactConfig)
    g = load("host_api")
    cfg, _ = _cfgs()
    cases = [
        lambda: DomainBounds(1.0, 0.0, 0.0, 1.0, 0.0, 1.0),
        lambda: DEMSolverConfig(DomainBounds(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), 0.0, Vector3(0.0, 0.0, 0.0),
                                HertzContactConfig(0.3, 0.3, 0.9, 0.9)),
        lambda: cfg.set_particle_properties(bogus=1.0),
        lambda: cfg.set_wall_properties(bogus=1.0),
        lambda: cfg.update_contact_model(bogus=1.0),
        lambda: HertzContactConfig(1.5, 0.3, 0.9, 0.9).validate(),
        lambda: HertzContactConfig(0.3, 0.3, 1.2, 0.9).validate(),
        lambda: LinearContactConfig(-1.0, 1.0, 0.1, 0.1, 0.3, 0.3).validate(),
        lambda: LinearContactConfig(1.0, 1.0, -0.1, 0.1, 0.3, 0.3).validate(),
        lambda: LinearContactConfig(1.0, 1.0, 0.1, 0.1, 0.3, 1.3).validate(),
    ]
    assert len(cases) == len(g["raises"])
    for fn, ref in zip(cases, g["raises"]):
        assert bool(ref)
        with pytest.raises(ValueError):
            fn()
