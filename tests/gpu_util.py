"""Builders shared by the GPU tests: the same scenarios as the golden
fixtures / oracle, constructed through the product's Python API."""
from lbdem_taichi_b200.cases import make_dem, rsa_spheres, rsa_spheres_grid  # noqa: F401
from lbdem_taichi_b200.dem3d.demconfig import HertzContactConfig, LinearContactConfig


def golden_dem(g, model):
    contact = (HertzContactConfig(pp_friction=0.3, pw_friction=0.4, pp_restitution=0.9, pw_restitution=0.8)
               if model == "hertz" else
               LinearContactConfig(stiffness_normal=200.0, stiffness_tangential=100.0, damping_normal=0.2,
                                   damping_tangential=0.1, pp_friction=0.3, pw_friction=0.4))
    return make_dem(g["domain"], float(g["dt"]), g["gravity"], contact, g["grad"], g["mass"], g["gpos"], g["gvel"],
                    omega=g["gomega"], periodic=tuple(bool(v) for v in g["periodic"]), E=float(g["E"]),
                    nu=float(g["nu"]), wall_E=float(g["wall_E"]), wall_nu=float(g["wall_nu"]),
                    max_coord=int(g["max_coord"]), model=model)
